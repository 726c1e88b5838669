"""Makes the golden vectors of tests/golden/ from the reference's own code, run here.

Inputs are small seeded synthetic batches (kache-hash_b200/synth.py); outputs come from the reference's describer and
table (kache-hash include/Kmer_Batch.hpp, include/Kmer_Lanes.hpp, include/Streaming_Kmer_Hash_Table.hpp), compiled
from its sources by oracle/Makefile into oracle/_ref/ (the AVX2 build, whose checksum is the non-AVX-512 variant).
Both inputs and outputs are stored, so the tests need neither the reference nor the generator's RNG.

    python tests/golden/make_golden.py
"""
import ctypes
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "kache-hash_b200"), os.path.join(ROOT, "tests")]

import numpy as np  # noqa: E402

import oracle  # noqa: E402
import synth  # noqa: E402
from kache import Batch  # noqa: E402


def ref_v3():
    L = ctypes.CDLL(os.path.join(oracle.REF_DIR, "libkache_ref_v3.so"))
    L.ref_describe.restype = ctypes.c_uint64
    L.ref_describe.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64] + [ctypes.c_void_p] * 6
    return L


def ragged(g, seed, n):
    rng = np.random.default_rng(seed)
    comp = bytes.maketrans(b"ACGTacgt", b"TGCAtgca")
    out = []
    for i in range(n):
        L_ = int(rng.integers(0, 400))
        st = int(rng.integers(0, len(g) - L_ + 1))
        s = bytearray(synth.ASCII[g[st:st + L_]].tobytes())
        if i % 4 == 1 and L_ > 8:
            for j in range(L_ // 4, L_ // 2):
                s[j] |= 0x20
        if i % 5 == 2 and L_ > 100:
            s[40], s[77] = ord("N"), ord("-")
        if i % 3 == 0:
            s = bytearray(bytes(s).translate(comp)[::-1])
        out.append(bytes(s))
    return out + [b"", b"ACGT", b"A" * 30, b"N" * 40, b"a" * 31, b"T" * 32, b"NNNNACGTACGTACGTACGTACGTACGTACGTACGTNNNN"]


def describe_golden():
    L = ref_v3()
    g = synth.genome(20_000, seed=101)
    b = Batch.of(ragged(g, 102, 120))
    out = {"bases": b.bases, "off": b.off}
    for k in (31, 27, 32):
        P = int(b.positions(k).sum())
        arrs = [np.zeros(max(P, 1), np.uint64), np.zeros(max(P, 1), np.uint64), np.zeros(max(P, 1), np.uint8),
                np.zeros(max(P, 1), np.uint8), np.zeros(max(P, 1), np.uint8), np.zeros(max(P, 1), np.uint64)]
        at = 0
        for i in range(b.n):
            s, e = int(b.off[i]), int(b.off[i + 1])
            if e - s < k:
                continue
            c = L.ref_describe(k, b.bases.ctypes.data + s, e - s, *[a.ctypes.data + at * a.itemsize for a in arrs])
            at += c
        for name, a in zip(("key", "h", "cs", "fwd", "valid", "h_lanes"), arrs):
            out[f"k{k}_{name}"] = a[:P]
    np.savez_compressed(os.path.join(HERE, "describe.npz"), **out)


def table_golden(name, k, vb, n, pow2, make_batches, op, x, oriented=False, x_rev=0):
    """Per-call inserted counts and capacities, the final sorted dump, and a lookup of the queries."""
    batches, queries = make_batches()
    R = oracle.RefTable(k, vb, n, 0.8, pow2, workers=2)
    u = R.register()
    ins, caps = [], []
    for b in batches:
        ins.append(R.insert_oriented(u, b, op, x, x_rev) if oriented else R.upsert(u, b, op, x))
        caps.append(R.capacity())
    keys, vals = R.dump()
    f, v, w = R.lookup(queries)
    out = {"k": k, "vb": vb, "n": n, "pow2": pow2, "op": op, "x": x, "x_rev": x_rev, "oriented": oriented,
           "ins": np.array(ins, np.uint64), "caps": np.array(caps, np.uint64), "keys": keys,
           "vals": vals if vals is not None else np.zeros(0, np.uint64), "q_found": f, "q_vals": v, "q_fwd": w,
           "q_bases": queries.bases, "q_off": queries.off, "size": R.size()}
    for i, b in enumerate(batches):
        out[f"b{i}_bases"], out[f"b{i}_off"] = b.bases, b.off
    out["nb"] = len(batches)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def main():
    describe_golden()
    g = synth.genome(40_000, seed=111)
    reads = Batch(*synth.reads_fixed(g, 240, 150, seed=112))

    def split(b, size):
        return [b.slice(i, min(i + size, b.n)) for i in range(0, b.n, size)]

    def map64():
        return split(reads, 13), Batch.of(ragged(g, 113, 60))
    table_golden("map64_resize", 31, 8, 10, False, map64, 16, 1)

    g32 = synth.genome(30_000, seed=121)
    pieces = Batch(*synth.stretches(g32, 150))

    def set32():
        return split(pieces, 17), Batch.of(ragged(g32, 122, 40))
    table_golden("set_k32_resize", 32, 0, 100, False, set32, 0, 0)

    g27 = synth.genome(30_000, seed=131)

    def or27():
        b = Batch.of(ragged(g27, 132, 200))
        return split(b, 13), Batch.of(ragged(g27, 133, 60))
    table_golden("u8_k27_oriented_or", 27, 1, 20_000, False, or27, 3, 1, oriented=True, x_rev=2)

    def u16_add():
        return split(reads, 40), Batch.of(ragged(g, 114, 30))
    table_golden("u16_add_saturating_pow2", 31, 2, 1000, True, u16_add, 2, 30000)


if __name__ == "__main__":
    main()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
