"""The oracle pinned: against the golden vectors the reference's own code produced (tests/golden/, made by
tests/golden/make_golden.py), against the reference's known answers (test/capi.cpp's sizing), and, where the
reference was built on this machine (oracle/_ref), against the live reference. CPU only."""
import glob
import os

import numpy as np
import pytest

import oracle
import synth
from kache import Batch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_describer_against_reference_golden():
    """describers.cpp: canonical key, minimizer hash, checksum, orientation per position, and the lane describer's
    minimizer hashes recomputed from keys, as the reference computed them."""
    z = np.load(os.path.join(GOLDEN, "describe.npz"))
    b = Batch(z["bases"], z["off"])
    o = oracle.oracle().L
    for k, l in ((31, 22), (27, 16), (32, 20)):
        key, h, cs, fwd, valid = oracle.describe(b, k, l)
        assert np.array_equal(valid, z[f"k{k}_valid"])
        for got, name in ((key, "key"), (h, "h"), (cs, "cs"), (fwd, "fwd")):
            assert np.array_equal(got, z[f"k{k}_{name}"]), (k, name)
        m = valid == 1
        assert m.sum() > 1000
        hl = np.array([o.orc_minimizer_hash(int(x), k, l) for x in key[m]], dtype=np.uint64)
        assert np.array_equal(hl, z[f"k{k}_h_lanes"][m])


def golden_tables():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")) if "describe" not in p)


@pytest.mark.parametrize("name", golden_tables())
def test_table_against_reference_golden(name):
    """Per-call inserted counts, the capacity after every call (resizes included), the sorted dump and lookups, as the
    reference's table gave them."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    k, vb, n, pow2, op, x = (int(z[f]) for f in ("k", "vb", "n", "pow2", "op", "x"))
    O = oracle.OracleTable(k, vb, n, 0.8, bool(pow2))
    u = O.register()
    for i in range(int(z["nb"])):
        b = Batch(z[f"b{i}_bases"], z[f"b{i}_off"])
        got = O.insert_oriented(u, b, op, x, int(z["x_rev"])) if bool(z["oriented"]) else O.upsert(u, b, op, x, x)
        assert got == z["ins"][i]
        assert O.capacity() == z["caps"][i]
    keys, vals = O.dump()
    assert O.size() == int(z["size"])
    assert np.array_equal(keys, z["keys"])
    if vb:
        assert np.array_equal(vals, z["vals"])
    q = Batch(z["q_bases"], z["q_off"])
    f, v, w = O.lookup(q)
    assert np.array_equal(f, z["q_found"]) and np.array_equal(w, z["q_fwd"])
    if vb:
        assert np.array_equal(v, z["q_vals"])


def test_sizing_known_answers():
    """capi.cpp:434-446: 1000 keys at 0.8 take 40 buckets (1280 slots), or 64 rounded to a power of 2; tables beyond
    2^32 - 1 buckets (2^31 rounded) are refused."""
    o = oracle.oracle().L
    assert o.orc_cap_for(1000, 0.8, 0) * 32 == 1280
    assert o.orc_cap_for(1000, 0.8, 1) * 32 == 2048
    assert o.orc_cap_for(1 << 22, 0.8, 0) == 163841
    assert not o.orc_fits(1 << 37, 0.8, 0)
    assert not o.orc_fits(55 << 30, 0.8, 1)
    assert not o.orc_fits(0xFFFFFFFFFFFFFFFF, 0.8, 0)
    assert o.orc_fits(1 << 22, 0.8, 0)


def test_known_hashes():
    """Wang's hash and the checksum on fixed values, computed by hand from their definitions (Kmer_Batch.hpp:24-67)."""
    o = oracle.oracle().L
    kat = {0: 0x77CFA1EEF01BCA90, 1: 0x5BCA7C69B794F8CE, 0x0123456789ABCDEF: 0x2A7C7E105D89D273,
           0xFFFFFFFFFFFFFFFF: 0x1F89206E3F8EC794}
    for x, h in kat.items():
        assert o.orc_wang(x) == h
    assert o.orc_checksum(0) == 1     # top byte 0 maps to 1
    assert o.orc_checksum(1) == 0x9E  # top byte of 0x9E3779B97F4A7C15
    assert o.orc_revcomp(0, 31) == (1 << 62) - 1
    assert o.orc_revcomp(0b00011011, 4) == 0b00011011   # ACGT is its own reverse complement


@pytest.mark.skipif(oracle.ref() is None, reason="the reference was not built on this machine")
@pytest.mark.parametrize("k,vb,n,pow2,op", [(31, 8, 10, False, 16), (31, 4, 5000, True, 2), (31, 0, 100, False, 0),
                                            (31, 1, 10, False, 16), (27, 1, 1000, False, 3), (32, 0, 50, False, 0)])
def test_oracle_against_live_reference(k, vb, n, pow2, op):
    g = synth.genome(100_000, seed=201)
    reads = Batch(*synth.reads_variable(g, 2, 150, 0.6, 30, 1200, seed=202))
    R = oracle.RefTable(k, vb, n, 0.8, pow2, workers=2)
    O = oracle.OracleTable(k, vb, n, 0.8, pow2)
    ur, uo = R.register(), O.register()
    for i in range(0, reads.n, 37):
        b = reads.slice(i, min(i + 37, reads.n))
        if k == 27:
            assert R.insert_oriented(ur, b, op, 1, 2) == O.insert_oriented(uo, b, op, 1, 2)
        else:
            assert R.upsert(ur, b, op, 1) == O.upsert(uo, b, op, 1, 1)
        assert R.capacity() == O.capacity()
    kr, vr = R.dump()
    ko, vo = O.dump()
    assert np.array_equal(kr, ko)
    if vb:
        assert np.array_equal(vr, vo)
    q = reads.slice(0, 200)
    fr, valr, wr = R.lookup(q)
    fo, valo, wo = O.lookup(q)
    assert np.array_equal(fr, fo) and np.array_equal(wr, wo)
    if vb:
        assert np.array_equal(valr, valo)
    if vb:
        for b in (reads.slice(0, 100), reads.slice(100, 300)):
            assert R.update(b, 16, 3) == O.update(b, 16, 3)
        assert np.array_equal(R.dump()[1], O.dump()[1])


@pytest.mark.skipif(oracle.ref() is None, reason="the reference was not built on this machine")
@pytest.mark.parametrize("k,n,lf,pow2", [(32, 1000, 0.8, False), (31, 300, 0.9, True)])
def test_capacity_replay_against_live_reference(k, n, lf, pow2):
    """The schedule replay used at full sizes (oracle.replay_capacity) gives the reference's capacity after each call
    from the call's inserted count alone."""
    g = synth.genome(300_000, seed=211)
    reads = Batch(*synth.reads_fixed(g, 6000, 150, seed=212))
    R = oracle.RefTable(k, 0, n, lf, pow2, workers=2)
    u = R.register()
    ins, caps = [], []
    for i in range(0, reads.n, 250):
        ins.append(R.upsert(u, reads.slice(i, min(i + 250, reads.n)), 0, 0))
        caps.append(R.capacity())
    assert list(oracle.replay_capacity(n, lf, pow2, ins)) == caps
    assert caps[-1] > caps[0]
