"""Lookups of prepared batch shapes (kache_b200_prepare_dev, kache_b200_lookup_prepared) through the C interface.

Each prepared lookup equals the staged lookup of the same batch (kache_b200_lookup_dev) bit for bit, and each prepared
count the staged count (kache_b200_count_dev), for fixed-length, ragged, odd (empty, short, non-ACGT, lowercase) and
empty batches. A run of them captured in a CUDA graph and replayed gives the same outputs, and again after the
batches' bases change in place (the same lengths, other k-mers). The table's epoch holds while queries run and changes
once an upsert grows the table.
"""
import numpy as np
import pytest

import kache
import synth
from kache import Batch

pytestmark = pytest.mark.gpu

K = 31


def _batches(g):
    fixed = Batch(*synth.reads_fixed(g, 3000, 150, seed=82))
    ragged = Batch(*synth.reads_variable(g, 0.5, 300, 1.0, 1, 3000, seed=83))
    odd = Batch.of([b"", b"ACGT", b"N" * 40, b"acgtNNacgt" * 9, b"C" * 31])
    return [fixed.slice(0, 256), fixed.slice(256, 1000), ragged.slice(0, min(ragged.n, 300)), odd, Batch.of([])]


def _on_device(b, dev):
    import torch
    bases = torch.from_numpy(np.concatenate([b.bases, np.zeros(16, np.uint8)])).to(dev)
    off = torch.from_numpy(b.off.view(np.int64).copy()).to(dev)
    return bases, off, b.n, int(b.positions(K).sum())


def _outputs(P, dev):
    import torch
    P = max(P, 1)
    return (torch.full((P,), 7, dtype=torch.uint8, device=dev), torch.zeros(P * 8, dtype=torch.uint8, device=dev),
            torch.full((P,), 7, dtype=torch.uint8, device=dev))


def _staged(T, db, dev):
    """kache_b200_lookup_dev of each batch, on the host."""
    import torch
    out = []
    for bases, off, n, P in db:
        f, v, w = _outputs(P, dev)
        T.lookup_dev(bases.data_ptr(), off.data_ptr(), n, f.data_ptr(), v.data_ptr(), w.data_ptr())
        torch.cuda.synchronize()
        out.append((f.cpu().numpy()[:P], v.cpu().numpy().view(np.uint64)[:P], w.cpu().numpy()[:P]))
    return out


def _staged_counts(T, db, dev):
    import torch
    out = []
    for bases, off, n, _ in db:
        c = torch.full((max(n, 1),), 99, dtype=torch.int64, device=dev)
        T.count_dev(bases.data_ptr(), off.data_ptr(), n, c.data_ptr())
        torch.cuda.synchronize()
        out.append(c.cpu().numpy().view(np.uint64)[:n])
    return out


def _counts(db, dev):
    import torch
    return [torch.full((max(n, 1),), 99, dtype=torch.int64, device=dev) for _, _, n, _ in db]


def _same_counts(cs, want, db):
    for c, w, (_, _, n, _) in zip(cs, want, db):
        assert np.array_equal(c.cpu().numpy().view(np.uint64)[:n], w)


def _same(outs, want, db):
    for (f, v, w), (wf, wv, ww), (_, _, _, P) in zip(outs, want, db):
        assert np.array_equal(f.cpu().numpy()[:P], wf)
        assert np.array_equal(v.cpu().numpy().view(np.uint64)[:P], wv)
        assert np.array_equal(w.cpu().numpy()[:P], ww)


def test_prepared_lookups_and_graph_replay():
    import torch
    dev = torch.device("cuda", 0)
    g = synth.genome(200_000, seed=81)
    T = kache.Table(K, 8, 100_000)
    u = T.register()
    T.upsert(u, Batch(*synth.reads_fixed(g, 4000, 150, seed=84)), kache.ADD_WRAP, 1, 1)
    db = [_on_device(b, dev) for b in _batches(g)]
    want = _staged(T, db, dev)
    want_c = _staged_counts(T, db, dev)
    assert any(int((f == 1).sum()) > 0 for f, _, _ in want)
    preps = [T.prepare_dev(off.data_ptr(), n) for _, off, n, _ in db]

    # One launch per batch, no staging.
    outs = [_outputs(P, dev) for _, _, _, P in db]
    cs = _counts(db, dev)
    for (bases, _, _, _), p, (f, v, w), c in zip(db, preps, outs, cs):
        T.lookup_prepared(p, bases.data_ptr(), f.data_ptr(), v.data_ptr(), w.data_ptr())
        T.count_prepared(p, bases.data_ptr(), c.data_ptr())
    torch.cuda.synchronize()
    _same(outs, want, db)
    _same_counts(cs, want_c, db)

    # The same launches captured in a CUDA graph on the table's stream, then replayed.
    e0 = T.epoch()
    outs = [_outputs(P, dev) for _, _, _, P in db]
    cs = _counts(db, dev)
    s = torch.cuda.Stream()
    T.set_stream(s.cuda_stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        for (bases, _, _, _), p, (f, v, w), c in zip(db, preps, outs, cs):
            T.lookup_prepared(p, bases.data_ptr(), f.data_ptr(), v.data_ptr(), w.data_ptr())
            T.count_prepared(p, bases.data_ptr(), c.data_ptr())
    torch.cuda.synchronize()
    assert all(int((f.cpu() == 7).sum()) == f.numel() for f, _, _ in outs)     # captured, not run
    graph.replay()
    torch.cuda.synchronize()
    _same(outs, want, db)
    _same_counts(cs, want_c, db)

    # Other bases of the same lengths (A->C->G->T->A, either case), written in place: the replay looks them up.
    lut = torch.arange(256, dtype=torch.uint8, device=dev)
    for a, b_ in ((65, 67), (67, 71), (71, 84), (84, 65), (97, 99), (99, 103), (103, 116), (116, 97)):
        lut[a] = b_
    for bases, _, _, _ in db:
        bases.copy_(lut[bases.long()])
    torch.cuda.synchronize()
    graph.replay()
    torch.cuda.synchronize()
    T.set_stream(None)
    want2 = _staged(T, db, dev)
    assert want2[0][0].tolist() != want[0][0].tolist()
    _same(outs, want2, db)
    _same_counts(cs, _staged_counts(T, db, dev), db)
    assert T.epoch() == e0

    # An upsert that grows the table moves its arrays: the epoch says so.
    cap = T.capacity()
    T.upsert(u, Batch(*synth.reads_fixed(synth.genome(400_000, seed=85), 8000, 150, seed=86)), kache.ADD_WRAP, 1, 1)
    assert T.capacity() > cap and T.epoch() != e0
    del graph
    for p in preps:
        T.prepared_free(p)
    T.close()


def test_prepared_validation():
    import torch
    dev = torch.device("cuda", 0)
    A = kache.Table(K, 8, 1000)
    B = kache.Table(K, 0, 1000)
    bases, off, n, P = _on_device(Batch.of([b"ACGT" * 20]), dev)
    f, v, w = _outputs(P, dev)
    pa = A.prepare_dev(off.data_ptr(), n)
    pb = B.prepare_dev(off.data_ptr(), n)
    with pytest.raises(kache.KacheError):
        B.lookup_prepared(pa, bases.data_ptr(), f.data_ptr())                   # another table's handle
    with pytest.raises(kache.KacheError):
        B.lookup_prepared(pb, bases.data_ptr(), f.data_ptr(), v.data_ptr())     # a set has no values
    with pytest.raises(kache.KacheError):
        A.lookup_prepared(pa, bases.data_ptr(), None)                           # no found array
    with pytest.raises(kache.KacheError):
        B.count_prepared(pa, bases.data_ptr(), f.data_ptr())                    # another table's handle
    with pytest.raises(kache.KacheError):
        A.count_prepared(pa, bases.data_ptr(), None)                            # no counts array
    A.lookup_prepared(pa, bases.data_ptr(), f.data_ptr(), v.data_ptr(), w.data_ptr())
    B.lookup_prepared(pb, bases.data_ptr(), f.data_ptr())
    torch.cuda.synchronize()
    A.prepared_free(pa), B.prepared_free(pb)
    A.close(), B.close()
