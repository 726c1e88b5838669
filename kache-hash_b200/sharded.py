"""One logical k-mer table over the ranks of a process group, one GPU per rank, partitioned by primary-bucket range.

The partition. A k-mer's primary bucket is ((h & 0xFFFFFFFF) * cap) >> 32 for its minimizer hash h
(include/Streaming_Kmer_Hash_Table.hpp:1015-1019), monotone in the low 32 bits of h at every capacity. Rank r of N
owns the k-mers with ((h & 0xFFFFFFFF) * N) >> 32 == r: a contiguous range of the logical table's buckets whatever
its capacity, and all k-mers of a super-k-mer (consecutive k-mers sharing a minimizer) have one owner. Secondary
buckets and overflow are the shard's own (placement is not observable).

One call, on every rank with its own batch:
  1. the batch is described on this rank (canonical keys, minimizer hashes, validity per position);
  2. each sequence is cut into runs: maximal stretches of consecutive valid positions with one owner;
  3. each run is sent as the bases it spans (its positions + k - 1), one buffer per owner, in one all-to-all
     (run lengths first, then bases): a k-mer's description depends on its own k bases only, so the owner
     re-describes the run exactly as the sender did;
  4. the owner runs the operation on its shard over the runs it received, as a batch of sequences;
  5. totals (keys inserted, k-mers present) are summed over the ranks (all-reduce); per-position results (lookups,
     and the per-sequence counts made from them) return by a second all-to-all, run by run, and are scattered into
     the requester's output positions. Positions that are not k-mers are answered on the requester.
Every rank takes the same collective steps in the same order. for_each is the concatenation of the shards' dumps;
size is the sum of the shards'.

The shard tables and the describer are given: kache.Table and its describer on the GPU (the default), or any objects
with their methods. The exchange goes through torch.distributed: with NCCL its buffers are staged on this rank's
current GPU, with gloo they stay in host memory; with one rank it is the plain table.
"""
import numpy as np

import kache


def owner_of(h, n):
    """The rank owning minimizer hashes h among n ranks: ((h & 0xFFFFFFFF) * n) >> 32."""
    h = np.asarray(h, dtype=np.uint64)
    return ((h & np.uint64(0xFFFFFFFF)) * np.uint64(n)) >> np.uint64(32)


def cut_runs(batch, k, h, valid, n):
    """The runs of a batch: maximal stretches of consecutive valid positions of one sequence with one owner.
    Returns (owner, seq, first position in the sequence, position count, first output index) per run, in output
    order; h and valid are per position in output order (sequence by sequence)."""
    pos = batch.positions(k)
    P = int(pos.sum())
    if P == 0:
        z = np.zeros(0, np.int64)
        return z, z, z, z, z
    seq = np.repeat(np.arange(batch.n, dtype=np.int64), pos)
    start = np.concatenate([[0], np.cumsum(pos)[:-1]]).astype(np.int64)
    within = np.arange(P, dtype=np.int64) - np.repeat(start, pos)
    own = owner_of(h, n).astype(np.int64)
    v = np.asarray(valid).astype(bool)
    # A run starts at a valid position whose predecessor is in another sequence, invalid or owned elsewhere, and ends
    # before the next start or invalid position.
    new = v.copy()
    new[1:] &= ~(v[:-1] & (seq[1:] == seq[:-1]) & (own[1:] == own[:-1]))
    first = np.flatnonzero(new)
    brk = np.flatnonzero(new | ~v)
    j = np.searchsorted(brk, first, side="right")
    end = np.where(j < len(brk), brk[np.minimum(j, len(brk) - 1)], P)
    return own[first], seq[first], within[first], end - first, first


class ShardedTable:
    """A k-mer table partitioned over the ranks of `group` (torch.distributed), one shard per rank.

    `make_shard()` returns this rank's shard table; `describe(batch)` returns (key, h, cs, fwd, valid) per position.
    Defaults: a kache.Table(k, value_bytes, expected_keys / ranks, load_factor, pow2) on this rank's GPU and its
    describer."""

    def __init__(self, k=31, value_bytes=8, expected_keys=1 << 22, load_factor=0.8, pow2=False, group=None,
                 make_shard=None, describe=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.n = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.k, self.vb = k, value_bytes
        per = max(1, -(-expected_keys // self.n))
        self.shard = make_shard() if make_shard else kache.Table(k, value_bytes, per, load_factor, pow2, capi=(k == 31))
        self.describe = describe or self.shard.describe
        self.user = self.shard.register()
        self._device = None

    def _dev(self):
        """Where the exchange's buffers live: this rank's current GPU under NCCL (which takes device tensors only),
        else host memory."""
        import torch
        if self._device is None:
            nccl = self.n > 1 and self.dist.get_backend(self.group) == "nccl"
            self._device = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")
        return self._device

    # ---- Exchange ------------------------------------------------------------------------------------------------

    def _all_to_all(self, parts, dtype):
        """Sends parts[r] (numpy arrays of dtype) to rank r; returns the arrays received from each rank."""
        import torch
        if self.n == 1:
            return [np.asarray(parts[0], dtype=dtype)]
        dev = self._dev()
        sizes = torch.tensor([len(p) for p in parts], dtype=torch.int64, device=dev)
        got = torch.empty(self.n, dtype=torch.int64, device=dev)
        self.dist.all_to_all_single(got, sizes, group=self.group)
        got = got.cpu().numpy()
        # Unsigned 64-bit words travel as signed ones (the bits unchanged): not every backend takes uint64.
        wire = np.int64 if np.dtype(dtype) == np.uint64 else dtype
        flat = np.concatenate([np.asarray(p, dtype=dtype) for p in parts]) if sum(map(len, parts)) else np.zeros(0, dtype)
        send = torch.from_numpy(np.ascontiguousarray(flat).view(wire)).to(dev)
        recv = torch.empty(int(got.sum()), dtype=send.dtype, device=dev)
        self.dist.all_to_all_single(recv, send, [int(x) for x in got], [len(p) for p in parts], group=self.group)
        r = recv.cpu().numpy().view(dtype)
        cuts = np.concatenate([[0], np.cumsum(got)])
        return [r[cuts[i]:cuts[i + 1]] for i in range(self.n)]

    def _sum(self, x):
        import torch
        if self.n == 1:
            return int(x)
        t = torch.tensor([int(x)], dtype=torch.int64, device=self._dev())
        self.dist.all_reduce(t, group=self.group)
        return int(t.item())

    def _route(self, b):
        """Describes batch b, cuts its runs and sends each to its owner. Returns (runs, the batch of runs this rank
        received, its per-source run counts, valid flags of b's positions)."""
        _, h, _, _, valid = self.describe(b)
        own, seq, p0, cnt, first = cut_runs(b, self.k, h, valid, self.n)
        lens = cnt + self.k - 1
        order = np.argsort(own, kind="stable")
        lens_parts, base_parts = [], []
        for r in range(self.n):
            sel = order[own[order] == r]
            lens_parts.append(lens[sel])
            starts = b.off[seq[sel]].astype(np.int64) + p0[sel]
            if len(sel):
                idx = np.repeat(starts, lens[sel]) + (np.arange(int(lens[sel].sum())) - np.repeat(np.concatenate([[0], np.cumsum(lens[sel])[:-1]]), lens[sel]))
                base_parts.append(b.bases[idx])
            else:
                base_parts.append(np.zeros(0, np.uint8))
        got_lens = self._all_to_all(lens_parts, np.int64)
        got_bases = self._all_to_all(base_parts, np.uint8)
        rl = np.concatenate(got_lens) if got_lens else np.zeros(0, np.int64)
        off = np.zeros(len(rl) + 1, np.uint64)
        np.cumsum(rl, out=off[1:])
        bases = np.concatenate(got_bases + [np.zeros(16, np.uint8)])
        runs = kache.Batch(bases, off)
        return (own, cnt, first, order), runs, [len(x) for x in got_lens], valid

    # ---- Operations -------------------------------------------------------------------------------------------------

    def upsert(self, b, op, x, init):
        """upsert over the logical table; returns the keys all ranks' calls inserted (the same on every rank)."""
        _, runs, _, _ = self._route(b)
        return self._sum(self.shard.upsert(self.user, runs, op, x, init) if runs.n else 0)

    def insert(self, b, op=kache.KEEP, x=0):
        _, runs, _, _ = self._route(b)
        return self._sum(self.shard.insert(self.user, runs, op, x) if runs.n else 0)

    def insert_oriented(self, b, op, x_fwd, x_rev):
        _, runs, _, _ = self._route(b)
        return self._sum(self.shard.insert_oriented(self.user, runs, op, x_fwd, x_rev, capi=False) if runs.n else 0)

    def update(self, b, op, x):
        _, runs, _, _ = self._route(b)
        return self._sum(self.shard.update(runs, op, x, capi=False) if runs.n else 0)

    def lookup(self, b):
        """Per-position (found, values as uint64, fwd) of b, laid out as kache_lookup's."""
        (own, cnt, first, order), runs, from_counts, valid = self._route(b)
        if runs.n:
            f, v, w = self.shard.lookup(runs, values=True, fwd=True)
            v = np.zeros(len(f), np.uint64) if v is None else v.astype(np.uint64)
        else:
            f, v, w = np.zeros(0, np.uint8), np.zeros(0, np.uint64), np.zeros(0, np.uint8)
        # Back to each run's sender, in the order it sent them.
        npos = runs.positions(self.k)
        cuts = np.concatenate([[0], np.cumsum(from_counts)])
        pcut = np.concatenate([[0], np.cumsum(npos)])
        back = [(f[pcut[cuts[r]]:pcut[cuts[r + 1]]], v[pcut[cuts[r]]:pcut[cuts[r + 1]]], w[pcut[cuts[r]]:pcut[cuts[r + 1]]])
                for r in range(self.n)]
        bf = np.concatenate(self._all_to_all([x[0] for x in back], np.uint8))
        bv = np.concatenate(self._all_to_all([x[1] for x in back], np.uint64))
        bw = np.concatenate(self._all_to_all([x[2] for x in back], np.uint8))
        P = int(b.positions(self.k).sum())
        found = np.where(np.asarray(valid).astype(bool), 0, 2).astype(np.uint8)
        values = np.zeros(P, np.uint64)
        fwd = np.zeros(P, np.uint8)
        # The results come back grouped by owner in send order: runs order[...] per owner.
        sent = np.concatenate([order[own[order] == r] for r in range(self.n)]) if len(own) else np.zeros(0, np.int64)
        if len(sent):
            idx = np.repeat(first[sent], cnt[sent]) + (np.arange(int(cnt[sent].sum())) - np.repeat(np.concatenate([[0], np.cumsum(cnt[sent])[:-1]]), cnt[sent]))
            found[idx], values[idx], fwd[idx] = bf, bv, bw
        return found, values, fwd

    def count(self, b):
        """Per-sequence counts of present k-mers (kache_count's)."""
        found, _, _ = self.lookup(b)
        pos = b.positions(self.k)
        hits = np.concatenate([[0], np.cumsum(found == 1)])
        ends = np.cumsum(pos)
        return (hits[ends] - hits[ends - pos]).astype(np.uint64)

    def size(self):
        return self._sum(self.shard.size())

    def dump(self):
        """The whole logical table's sorted (keys, values), on every rank: the shards' dumps concatenated."""
        import torch
        keys, vals = self.shard.dump()
        vals = np.zeros(len(keys), np.uint64) if vals is None else vals.astype(np.uint64)
        if self.n == 1:
            return keys, (vals if self.vb else None)
        out = [None] * self.n
        self.dist.all_gather_object(out, (keys, vals), group=self.group)
        k = np.concatenate([o[0] for o in out])
        v = np.concatenate([o[1] for o in out])
        o = np.argsort(k, kind="stable")
        return k[o], (v[o] if self.vb else None)
