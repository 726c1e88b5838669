"""The C interface against the reference's own C interface library (capi/*.cpp, compiled by oracle/Makefile's `capi`
target into oracle/_ref/libkache_capi_ref.so), the same call sequence through both libraries in one process:

- without a GPU: every status code for bad arguments that is decided before any table work (kache_new's options,
  null tables and pointers), kache_supports, kache_default_options, kache_strerror;
- on the GPU: bad arguments on live tables (users, ops, null batches and outputs), inserts of every op and width,
  oriented inserts, updates, per-sequence counts / masked counts / sums, per-position lookups, single-k-mer gets,
  reductions of each kind with masks and worker counts, for_each's chunks (at most 4,096 keys, 2-bit MSB-first
  encoding, values, early stop) over shares, sizes, kache_get_stats' capacity, and the 129th user."""
import ctypes

import numpy as np
import pytest

import kache
import oracle
import synth
from kache import Batch

_vp = ctypes.c_void_p


def ref():
    R = oracle.ref_capi()
    if R is None:
        pytest.skip("the reference's C interface library (oracle/_ref/libkache_capi_ref.so) is not built")
    return R


def both():
    return kache.lib(), ref()


def test_supports_defaults_strerror_alike():
    L, R = both()
    for k in (0, 21, 27, 31, 32, 63):
        for w in (0, 1, 2, 3, 4, 5, 8, 16):
            assert bool(L.kache_supports(k, w)) == bool(R.kache_supports(k, w)), (k, w)
            a, b = L.kache_default_options(k, w), R.kache_default_options(k, w)
            assert (a.k, a.value_bytes, a.expected_keys, a.load_factor, a.resize_workers, a.pow2_capacity) == \
                   (b.k, b.value_bytes, b.expected_keys, b.load_factor, b.resize_workers, b.pow2_capacity), (k, w)
    for c in list(range(-2, 7)) + [99]:
        assert L.kache_strerror(c) == R.kache_strerror(c), c


def _options(L, **kw):
    o = L.kache_default_options(31, 4)
    for f, v in kw.items():
        setattr(o, f, v)
    return o


BAD_OPTIONS = [dict(k=25), dict(value_bytes=3), dict(value_bytes=16), dict(load_factor=0.0), dict(load_factor=1.0),
               dict(load_factor=1.5), dict(load_factor=float("nan")), dict(load_factor=-0.5), dict(resize_workers=0),
               dict(pow2_capacity=2), dict(expected_keys=1 << 37), dict(expected_keys=55 << 30, pow2_capacity=1),
               dict(expected_keys=0xFFFFFFFFFFFFFFFF)]


@pytest.mark.parametrize("kw", BAD_OPTIONS, ids=[",".join(f"{k}={v}" for k, v in d.items()) for d in BAD_OPTIONS])
def test_new_rejections_alike(kw):
    L, R = both()
    codes = []
    for lib in (L, R):
        h = _vp()
        o = _options(lib, **kw)
        codes.append((lib.kache_new(ctypes.byref(o), ctypes.byref(h)), bool(h.value)))
        if h.value:
            lib.kache_free(h)
    assert codes[0] == codes[1]
    for lib in (L, R):
        o = _options(lib)
        assert lib.kache_new(ctypes.byref(o), None) == lib.kache_new(None, None)


def test_null_table_calls_alike():
    L, R = both()
    u, x = ctypes.c_uint32(), ctypes.c_uint64()
    st = kache.Stats()
    f, v = ctypes.c_uint8(), ctypes.c_uint64()
    fn = kache.KEYS_FN(lambda ctx, keys, vals, n: 0)
    for lib in (L, R):
        lib.kache_free(None)
    calls = [
        lambda l: l.kache_register(None, ctypes.byref(u)),
        lambda l: l.kache_insert(None, 0, None, None, 0, 0, 0, ctypes.byref(x)),
        lambda l: l.kache_insert_oriented(None, 0, None, None, 0, 0, 0, 0, ctypes.byref(x)),
        lambda l: l.kache_update(None, None, None, 0, 0, 0, ctypes.byref(x)),
        lambda l: l.kache_count(None, None, None, 0, None),
        lambda l: l.kache_count_masked(None, None, None, 0, 1, 1, None),
        lambda l: l.kache_sum(None, None, None, 0, None),
        lambda l: l.kache_lookup(None, None, None, 0, None, None, None),
        lambda l: l.kache_get(None, b"A" * 31, ctypes.byref(f), ctypes.byref(v)),
        lambda l: l.kache_size(None, ctypes.byref(x)),
        lambda l: l.kache_reduce(None, 0, 1, 1, ctypes.byref(x)),
        lambda l: l.kache_for_each(None, 1, 0, fn, None),
        lambda l: l.kache_get_stats(None, ctypes.byref(st)),
    ]
    for i, c in enumerate(calls):
        assert c(L) == c(R), i


# ---- On the GPU: the same calls on live tables ------------------------------------------------------------------

class Pair:
    """One table in each library, made with the same options."""

    def __init__(self, vb, n=200_000, lf=0.8, pow2=0):
        self.L, self.R = both()
        self.vb = vb
        self.h = []
        for lib in (self.L, self.R):
            h = _vp()
            o = _options(lib, value_bytes=vb, expected_keys=n, load_factor=lf, pow2_capacity=pow2)
            assert lib.kache_new(ctypes.byref(o), ctypes.byref(h)) == kache.KACHE_OK
            self.h.append(h)

    def close(self):
        for lib, h in zip((self.L, self.R), self.h):
            lib.kache_free(h)

    def call(self, name, *args):
        """Calls `name(table, *args)` in both libraries (an argument given as a function of the library's index 0 or
        1 is evaluated per library: its outputs); returns both statuses."""
        out = []
        for i, (lib, h) in enumerate(zip((self.L, self.R), self.h)):
            a = [x(i) if callable(x) else x for x in args]
            out.append(getattr(lib, name)(h, *a))
        return out

    def register(self):
        us = [ctypes.c_uint32(), ctypes.c_uint32()]
        codes = self.call("kache_register", lambda i: ctypes.byref(us[i]))
        return codes, [u.value for u in us]


@pytest.mark.gpu
@pytest.mark.parametrize("vb", [0, 1, 2, 4, 8])
def test_operations_alike(vb):
    g = synth.genome(100_000, seed=61)
    b1 = Batch(*synth.reads_fixed(g, 3000, 150, seed=62))
    b2 = Batch(*synth.reads_variable(g, 0.5, 150, 1.0, 1, 3000, seed=63))
    q = Batch(*synth.reads_variable(g, 0.3, 150, 1.0, 1, 3000, seed=64))
    P = Pair(vb)
    codes, (u0, u1) = P.register()
    assert codes == [0, 0] and u0 == u1 == 0
    vt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}.get(vb, np.uint8)
    mx = (1 << (8 * vb)) - 1 if vb else 0

    # Bad arguments on a live table: unregistered users, unknown ops, null batches and outputs.
    x = [ctypes.c_uint64(), ctypes.c_uint64()]
    for user, op, args in ((7, 0, b1.args()), (0, 6, b1.args()), (0, 99, b1.args()), (0, 0, (None, None, 3))):
        assert len(set(P.call("kache_insert", user, *args, op, 1, lambda i: ctypes.byref(x[i])))) == 1, (user, op)
    assert len(set(P.call("kache_insert", 0, *b1.args(), 0, 1, None))) == 1
    assert len(set(P.call("kache_count", *b1.args(), None))) == 1
    assert len(set(P.call("kache_lookup", *q.args(), None, None, None))) == 1
    assert len(set(P.call("kache_update", *b1.args(), 7, 1, lambda i: ctypes.byref(x[i])))) == 1

    # Inserts: every op in turn (commutative within a call, so the results are deterministic), growth included.
    for bb, op, val in ((b1, kache.ADD, 3), (b2, kache.MAX, 9), (b1, kache.OR, 0x50), (b2, kache.ADD, mx), (b1, kache.MIN, 2),
                        (b2, kache.KEEP, 1), (b1, kache.ASSIGN, 7)):
        r = P.call("kache_insert", 0, *bb.args(), op, val, lambda i: ctypes.byref(x[i]))
        assert r[0] == r[1], (op, val)
        if r[0] == 0:
            assert x[0].value == x[1].value, (op, val)
    r = P.call("kache_insert_oriented", 0, *b2.args(), kache.OR, 1, 2, lambda i: ctypes.byref(x[i]))
    assert r[0] == r[1] and (r[0] != 0 or x[0].value == x[1].value)
    r = P.call("kache_update", *q.args(), kache.ADD, 5, lambda i: ctypes.byref(x[i]))
    assert r[0] == r[1] and (r[0] != 0 or x[0].value == x[1].value)

    # Queries.
    n = q.n
    for name, extra in (("kache_count", ()), ("kache_count_masked", (0x3, 0x50)), ("kache_sum", ())):
        outs = [np.full(n, 77, np.uint64), np.full(n, 77, np.uint64)]
        r = P.call(name, *q.args(), *extra, lambda i: outs[i].ctypes.data)
        assert r[0] == r[1], name
        if r[0] == 0:
            assert np.array_equal(outs[0], outs[1]), name
    pos = int(q.positions(31).sum())
    fo = [np.full(pos, 9, np.uint8) for _ in range(2)]
    vo = [np.full(pos, 0xAB, vt) for _ in range(2)]
    wo = [np.full(pos, 9, np.uint8) for _ in range(2)]
    r = P.call("kache_lookup", *q.args(), lambda i: fo[i].ctypes.data, lambda i: vo[i].ctypes.data if vb else None,
               lambda i: wo[i].ctypes.data)
    assert r == [0, 0]
    assert np.array_equal(fo[0], fo[1]) and np.array_equal(wo[0], wo[1])
    if vb:
        assert np.array_equal(vo[0], vo[1])
    f, v = [ctypes.c_uint8(), ctypes.c_uint8()], [ctypes.c_uint64(), ctypes.c_uint64()]
    rng = np.random.default_rng(65)
    acgt = np.frombuffer(b"ACGTNacgt", np.uint8)
    for s in rng.integers(0, len(g) - 31, 300):
        kmer = np.frombuffer(b"ACGT", np.uint8)[g[int(s):int(s) + 31]].tobytes()
        for variant in (kmer, kmer.lower(), kmer[:10] + b"N" + kmer[11:], acgt[rng.integers(0, 9, 31)].tobytes()):
            r = P.call("kache_get", variant, lambda i: ctypes.byref(f[i]), lambda i: ctypes.byref(v[i]))
            assert r[0] == r[1] and (f[0].value, v[0].value) == (f[1].value, v[1].value), variant
    r = P.call("kache_size", lambda i: ctypes.byref(x[i]))
    assert r == [0, 0] and x[0].value == x[1].value

    # Reductions of each kind, masks and worker counts.
    for what in (0, 1, 2, 3):
        for mask in (0xFFFFFFFFFFFFFFFF, 0x1, 0x50, 0):
            for workers in (1, 4, 0):
                r = P.call("kache_reduce", what, mask, workers, lambda i: ctypes.byref(x[i]))
                assert r[0] == r[1], (what, mask, workers)
                if r[0] == 0:
                    assert x[0].value == x[1].value, (what, mask, workers)

    # for_each: shares, chunks, encoding, values, early stop.
    for shards in (1, 3, 0):
        got = []
        for i in range(2):
            keys, vals, sizes = [], [], []

            def cb(ctx, kp, vp, cnt, keys=keys, vals=vals, sizes=sizes):
                sizes.append(cnt)
                keys.append(np.ctypeslib.as_array(kp, shape=(cnt,)).copy())
                if vp:
                    vals.append(np.ctypeslib.as_array(ctypes.cast(vp, ctypes.POINTER(np.ctypeslib.as_ctypes_type(vt))), shape=(cnt,)).copy())
                return 0

            fn = kache.KEYS_FN(cb)
            lib = (P.L, P.R)[i]
            codes = [lib.kache_for_each(P.h[i], shards, s, fn, None) for s in range(max(shards, 1))]
            k_ = np.concatenate(keys) if keys else np.zeros(0, np.uint64)
            v_ = np.concatenate(vals) if vals else None
            o = np.argsort(k_)
            got.append((codes, k_[o], None if v_ is None else v_[o], max(sizes, default=0), bool(vals)))
        assert got[0][0] == got[1][0], shards
        if all(c == 0 for c in got[0][0]):
            assert np.array_equal(got[0][1], got[1][1])
            assert got[0][4] == got[1][4]
            if got[0][2] is not None:
                assert np.array_equal(got[0][2], got[1][2])
            assert got[0][3] <= 4096 and got[1][3] <= 4096
    stops = []
    for i in range(2):
        calls = []
        fn = kache.KEYS_FN(lambda ctx, kp, vp, cnt: calls.append(cnt) or 1)
        (P.L, P.R)[i].kache_for_each(P.h[i], 1, 0, fn, None)
        stops.append(len(calls))
    assert stops == [1, 1]

    st = [kache.Stats(), kache.Stats()]
    assert P.call("kache_get_stats", lambda i: ctypes.byref(st[i])) == [0, 0]
    assert st[0].capacity == st[1].capacity and st[0].keys == st[1].keys
    P.close()


@pytest.mark.gpu
def test_users_alike():
    """kache_register hands out users 0..127, then fails alike (capi/kache_capi.cpp:117-135)."""
    P = Pair(4, 1000)
    for expect in range(128):
        codes, us = P.register()
        assert codes == [0, 0] and us == [expect, expect]
    codes, _ = P.register()
    assert codes[0] == codes[1] == kache.KACHE_EUSERS
    P.close()


@pytest.mark.gpu
def test_capacity_alike_across_growth():
    """kache_get_stats' capacity after every insert of a table that grows (exact and power-of-2 sizing), one user."""
    g = synth.genome(400_000, seed=66)
    b = Batch(*synth.reads_fixed(g, 12_000, 150, seed=67))
    for pow2 in (0, 1):
        P = Pair(8, 20_000, 0.8, pow2)
        P.register()
        st = [kache.Stats(), kache.Stats()]
        x = [ctypes.c_uint64(), ctypes.c_uint64()]
        for s in range(0, b.n, 1000):
            p = b.slice(s, min(b.n, s + 1000))
            assert P.call("kache_insert", 0, *p.args(), kache.ADD, 1, lambda i: ctypes.byref(x[i])) == [0, 0]
            assert x[0].value == x[1].value
            P.call("kache_get_stats", lambda i: ctypes.byref(st[i]))
            assert st[0].capacity == st[1].capacity, (pow2, s)
        P.close()
