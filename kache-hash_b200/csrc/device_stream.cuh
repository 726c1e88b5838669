// The warp describer and the streaming kernel: one warp describes a segment of a sequence, 32 k-mer positions per
// row, and hands each row's k-mers to a visitor (upsert, update, lookup, count, ...), one k-mer per lane.
//
// What it computes per position is the reference describers' description (include/Kmer_Batch.hpp:191-250,
// include/Kmer_Lanes.hpp:164-244): the canonical key, its orientation, its checksum and its l-minimizer hash. How:
//   - each row of 32 bases is loaded coalesced (lane j reads base j), turned into 2-bit codes and an ACGT bit, and
//     packed by warp OR-reductions into a forward word W (first base most significant) and a complemented word R
//     (first base least significant), once per row rather than once per k-mer;
//   - lane j's k-mer is a 2k-bit funnel window of (W_r, W_r+1) and its reverse complement one of (R_r, R_r+1);
//   - each lane hashes the l-mer at its position; the minima of neighbouring pairs of those hashes go to a per-warp
//     ring in shared memory, and a k-mer's minimizer hash, the least of the w = k - l + 1 hashes from its own position
//     on, is the least of ceil(w / 2) pair minima;
//   - non-ACGT characters split sequences (DNA_Utility.hpp:199-224): a window with one is not a k-mer.
// Sequences are cut into segments of up to `seg_positions` positions; each segment re-reads the k - 1 bases it
// shares with the next, so segments, like the reference's lanes (include/Streaming_Kmer_Hash_Table.hpp:1751-1781),
// need no state from one another.
#pragma once

#include "device_table.cuh"

namespace kache_b200
{

// A batch on the device: sequence q is bases[off[q], off[q+1]); segs lists (q << 24 | s) for the s'th segment, of
// seg_len positions, of each sequence of at least k bases; pos_off[q] counts the positions of the sequences before q.
// With seq_addr set (several batches run as one), off only lays the lengths end to end and sequence q's
// off[q+1] - off[q] bases are read at the device address seq_addr[q], where its own batch holds them.
struct Dev_Batch
{
    const uint8_t* bases;
    const uint64_t* off;
    const uint64_t* segs;
    const uint64_t* pos_off;
    uint64_t n;
    uint64_t nsegs;
    uint32_t seg_len;   // A multiple of 32.
    const uint64_t* seq_addr = nullptr;

    __device__ __forceinline__ const uint8_t* seq(const uint64_t q, const uint64_t b0) const
    {
        return seq_addr ? reinterpret_cast<const uint8_t*>(seq_addr[q]) : bases + b0;
    }
};

constexpr int stream_warps = 8;

// One row of 32 bases, packed.
struct Row
{
    uint64_t W, R;
    uint32_t valid;
};

// The row at offset o of a segment, through this lane's base pointer sp (the segment's first base + lane) and its
// bound rem (the sequence's bases from sp on, capped at 2^30): 32-bit arithmetic per row.
__device__ __forceinline__ Row load_row(const uint8_t* sp, const int32_t rem, const uint32_t o, const uint32_t lane)
{
    constexpr uint32_t all = 0xFFFFFFFFu;
    const uint32_t ch = static_cast<int32_t>(o) < rem ? sp[o] : 0u;
    const uint32_t x = (ch | 0x20u) - 'a';
    const bool ok = x < 20u && ((0x80045u >> x) & 1u);     // a, c, g, t
    const uint32_t code = ((ch >> 2) ^ (ch >> 1)) & 3u;
    const bool first = lane < 16;
    const uint32_t s = 2 * (lane & 15);
    const uint32_t f = code << (30 - s), z = code << s;
    Row r;
    r.valid = __ballot_sync(all, ok);
    // Base j at bits 63 - 2j .. 62 - 2j of W, and at bits 2j .. 2j + 1 of ~R.
    const uint32_t w_hi = __reduce_or_sync(all, first ? f : 0u), w_lo = __reduce_or_sync(all, first ? 0u : f);
    const uint32_t z_lo = __reduce_or_sync(all, first ? z : 0u), z_hi = __reduce_or_sync(all, first ? 0u : z);
    r.W = (uint64_t(w_hi) << 32) | w_lo;
    r.R = ~((uint64_t(z_hi) << 32) | z_lo);
    return r;
}

// The forward and reverse-complement n-mers (n <= 32) starting at base j of row a, spilling into row b: 64-bit
// windows of the 128-bit pairs (a.W, b.W) and (b.R, a.R) at bit offset 2j, as two 32-bit funnel shifts each; which
// words feed them depends on the lane only (j >= 16).
template <int n>
__device__ __forceinline__ void window(const Row& a, const Row& b, const uint32_t j, uint64_t& f, uint64_t& r)
{
    const bool big = j >= 16;
    const uint32_t sh = (2 * j) & 31;
    const uint32_t a1 = static_cast<uint32_t>(a.W >> 32), a0 = static_cast<uint32_t>(a.W);
    const uint32_t b1 = static_cast<uint32_t>(b.W >> 32), b0 = static_cast<uint32_t>(b.W);
    const uint32_t x3 = big ? a0 : a1, x2 = big ? b1 : a0, x1 = big ? b0 : b1;
    const uint64_t top = (uint64_t(__funnelshift_l(x2, x3, sh)) << 32) | __funnelshift_l(x1, x2, sh);
    f = top >> (64 - 2 * n);
    const uint32_t r0 = static_cast<uint32_t>(a.R), r1 = static_cast<uint32_t>(a.R >> 32);
    const uint32_t r2 = static_cast<uint32_t>(b.R), r3 = static_cast<uint32_t>(b.R >> 32);
    const uint32_t y0 = big ? r1 : r0, y1 = big ? r2 : r1, y2 = big ? r3 : r2;
    const uint64_t low = (uint64_t(__funnelshift_r(y1, y2, sh)) << 32) | __funnelshift_r(y0, y1, sh);
    r = low & kmer_mask(n);
}

// A k-mer as the visitors get it.
struct Kmer_Desc
{
    uint64_t key, h;
    uint64_t q, pos;    // Sequence and position in it.
    uint64_t out;       // Index of the position in the batch's outputs (set by the lane kernel; 0 in the warp kernel).
    uint8_t c;
    bool fwd;           // Occurs as its canonical form.
    bool valid;         // All k characters are ACGT.
    bool in;            // The position exists (is in the segment).
    bool last;          // Unused; false.
};

template <int k, int l, typename Visitor>
__global__ void __launch_bounds__(32 * stream_warps) stream_kernel(const Dev_Batch batch, const uint64_t seg_b, const uint64_t seg_e, Visitor vis)
{
    constexpr int w = k - l + 1;
    static_assert(k <= 32 && l < k && w <= 32, "k-mers in a machine word, minimizers of at least two l-mers");
    constexpr uint32_t all = 0xFFFFFFFFu;
    // Pair minima: entry 32 (r & 1) + j is min(H[i - 1], H[i]) for position i = 32 r + j of the segment, where H are
    // the l-mer hashes; rows r and r + 1 are held.
    __shared__ uint64_t ring_all[stream_warps][64];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t* ring = ring_all[wid];
    vis.begin();

    const uint64_t warps = uint64_t(gridDim.x) * stream_warps;
    for(uint64_t g = seg_b + uint64_t(blockIdx.x) * stream_warps + wid; g < seg_e; g += warps)
    {
        const uint64_t packed = batch.segs[g];
        const uint64_t q = packed >> 24, s = packed & 0xFFFFFF;
        const uint64_t b0 = batch.off[q], len = batch.off[q + 1] - b0;
        const uint8_t* seq = batch.seq(q, b0);
        const uint64_t npos = len - k + 1;
        const uint64_t p0 = s * batch.seg_len;
        const uint64_t p1 = min(npos, p0 + batch.seg_len);
        const uint32_t rows = static_cast<uint32_t>((p1 - p0 + 31) / 32);
        const uint32_t in_seg = static_cast<uint32_t>(p1 - p0);
        const uint8_t* sp = seq + p0 + lane;
        const int32_t rem = static_cast<int32_t>(min(len - p0, uint64_t(1) << 30)) - static_cast<int32_t>(lane);

        Row r0 = load_row(sp, rem, 0, lane);
        Row r1 = load_row(sp, rem, 32, lane);
        uint64_t hprev;     // This lane's l-mer hash in the newest row hashed.
        {
            uint64_t f, rc;
            window<l>(r0, r1, lane, f, rc);
            hprev = wang_u64(f < rc ? f : rc);
            const uint64_t left = __shfl_up_sync(all, hprev, 1);
            ring[lane] = lane ? min64(left, hprev) : hprev;  // Entry 0 is never read.
        }

        vis.begin_segment(q);
        for(uint32_t r = 0; r < rows; ++r)
        {
            const Row r2 = load_row(sp, rem, 32 * (r + 2), lane);
            {
                uint64_t f, rc;
                window<l>(r1, r2, lane, f, rc);
                const uint64_t hc = wang_u64(f < rc ? f : rc);
                const uint64_t up = __shfl_up_sync(all, hc, 1), last = __shfl_sync(all, hprev, 31);
                ring[((r + 1) & 1) * 32 + lane] = min64(lane ? up : last, hc);
                hprev = hc;
            }
            __syncwarp();

            Kmer_Desc d;
            uint64_t f, rc;
            window<k>(r0, r1, lane, f, rc);
            // ACGT flags of the 32 bases from this lane's position on (k <= 32 of them make its k-mer).
            const uint32_t vbits = __funnelshift_r(r0.valid, r1.valid, lane);
            constexpr uint32_t km = (k == 32 ? 0xFFFFFFFFu : (1u << k) - 1);
            d.pos = p0 + 32 * r + lane;
            d.out = 0, d.last = false;
            d.q = q;
            d.in = 32 * r + lane < in_seg;
            d.valid = d.in && (vbits & km) == km;
            d.key = f < rc ? f : rc;
            d.fwd = f <= rc;
            d.c = checksum_of(d.key);
            // Pairs (i - 1, i) at i = j + 1, j + 3, ...: w / 2 of them cover [j, j + w - 1] for even w; for odd w the
            // pair at j + w - 1 adds the last hash.
            uint64_t h = ~0ull;
            const uint32_t base = (r & 1) * 32 + lane;
#pragma unroll
            for(int o = 1; o < w; o += 2)
                h = min64(h, ring[(base + o) & 63]);
            if constexpr(w % 2 == 1)
                h = min64(h, ring[(base + w - 1) & 63]);
            d.h = h;

            vis.visit(d, lane);
            __syncwarp();
            r0 = r1, r1 = r2;
        }
        vis.end_segment(q, lane);
    }
    vis.end(lane);
}

// ---- Visitors -------------------------------------------------------------------------------------------------

// Per-warp counter flush: one atomic per warp at the end of the kernel.
__device__ __forceinline__ void warp_flush(unsigned long long* ctr, const unsigned long long c, const uint32_t lane)
{
    if(lane == 0 && c)
        atomicAdd(ctr, c);
}

// Upsert / insert / upsert_oriented (include/Streaming_Kmer_Hash_Table.hpp:2219-2514): returns the keys inserted;
// k-mers that found the overflow table full set their bit in `retry_out` and change nothing. In retry mode, only
// the positions whose bit is set in `retry_in` run.
template <bool set_, typename V, typename Fn>
struct Upsert_Visitor
{
    Dev_Table T;
    Fn fn;
    const uint64_t* pos_off;
    unsigned long long* inserted;
    unsigned int* retry_out;
    const unsigned int* retry_in;
    unsigned int* retried;      // Set to 1 if any bit of retry_out was set.
    unsigned long long ins;
    unsigned long long* per_seq;    // If set, keys inserted per sequence are added at per_seq[q] (lane kernel only).
    uint32_t lane_ins;
    static constexpr int stage_bytes = 0;

    // No checksum cache for inserts: other lanes insert into the same buckets meanwhile, and a stale copy's missed
    // candidates cost a re-read; measured slower than reading the sector each time (config-1 upsert 1.91 vs 1.74 ms).
    __device__ __forceinline__ void lane_cache(uint4*, uint4*) {}

    __device__ __forceinline__ void begin() { ins = 0; }
    __device__ __forceinline__ void begin(uint8_t*) { ins = 0; }
    __device__ __forceinline__ void begin_segment(uint64_t) {}
    __device__ __forceinline__ void end_segment(uint64_t, uint32_t) {}
    __device__ __forceinline__ void lane_begin(uint64_t, bool) { lane_ins = 0; }
    __device__ __forceinline__ void lane_end(const uint64_t q, const bool has)
    {
        if(per_seq && has && lane_ins)
            atomicAdd(per_seq + q, static_cast<unsigned long long>(lane_ins));
    }

    __device__ __forceinline__ void visit(const Kmer_Desc& d, const uint32_t lane)
    {
        bool active = d.valid;
        if(retry_in && active)
        {
            const uint64_t gpos = d.out;
            active = (retry_in[gpos >> 5] >> (gpos & 31)) & 1;
        }

        Landing L{};
        uint32_t r = NONE;
        if(active)
            r = upsert_chain<set_>(T, d.key, d.h, d.c, L);
        const bool comm = fn.commutes();
        if(r == INSERTED)
        {
            if constexpr(!set_)
            {
                if(comm)
                    fn.apply_init(L.val, d.fwd);
                else
                    write_val<V>(L.val, fn.initial(d.fwd));
            }
            publish(L, !set_ && !comm);
        }
        else if(r == OV_FULL)
        {
            const uint64_t gpos = d.out;
            atomicOr(retry_out + (gpos >> 5), 1u << (gpos & 31));
            *retried = 1;
        }
        ins += __popc(__ballot_sync(0xFFFFFFFFu, r == INSERTED));
        lane_ins += (r == INSERTED);
        __syncwarp();

        if constexpr(!set_)
            if((r == FOUND || r == FOUND_PENDING) && !fn.is_noop())
            {
                if(r == FOUND_PENDING && !comm && !await_published(L, T.wait_polls))
                    atomicOr(T.err, ERR_WAIT);
                fn.apply(L.val, d.fwd);
            }
        if(r == INSERTED && !L.cs)
            atomicAdd(T.ov_count, 1ull);
    }

    __device__ __forceinline__ void end(const uint32_t lane) { warp_flush(inserted, ins, lane); }
};

// Present-only update (include/Streaming_Kmer_Hash_Table.hpp:2650-2691): returns the k-mers present, repeats counted.
template <typename V, typename Fn>
struct Update_Visitor
{
    Dev_Table T;
    Fn fn;
    unsigned long long* present;
    unsigned long long cnt;
    Bucket_Cache bc;            // Bound by the lane kernel (exact: an update inserts nothing); unbound elsewhere.
    unsigned long long* per_seq = nullptr;  // If set, k-mers present per sequence are added at per_seq[q] (lane kernel).
    uint32_t lane_cnt = 0;
    static constexpr int stage_bytes = 0;

    __device__ __forceinline__ void lane_cache(uint4* lo, uint4* hi) { bc.lo = lo, bc.hi = hi, bc.b = ~0ull; }

    __device__ __forceinline__ void begin() { cnt = 0; }
    __device__ __forceinline__ void begin(uint8_t*) { cnt = 0; }
    __device__ __forceinline__ void begin_segment(uint64_t) {}
    __device__ __forceinline__ void end_segment(uint64_t, uint32_t) {}
    __device__ __forceinline__ void lane_begin(uint64_t, bool) { lane_cnt = 0; }
    __device__ __forceinline__ void lane_end(const uint64_t q, const bool has)
    {
        if(per_seq && has && lane_cnt)
            atomicAdd(per_seq + q, static_cast<unsigned long long>(lane_cnt));
    }

    __device__ __forceinline__ void visit(const Kmer_Desc& d, const uint32_t)
    {
        unsigned long long* v = nullptr;
        if(d.valid)
            v = find_chain<false, true>(T, d.key, d.h, d.c, bc.lo ? &bc : nullptr);
        if(v)
            fn.apply(v, d.fwd);
        cnt += __popc(__ballot_sync(0xFFFFFFFFu, v != nullptr));
        lane_cnt += (v != nullptr);
    }

    __device__ __forceinline__ void end(const uint32_t lane) { warp_flush(present, cnt, lane); }
};

// Per-position lookup (capi/Kmer_Table.hpp:163-190): found (0 absent, 1 present, 2 not a k-mer), value, orientation
// at pos_off[q] + i.
template <bool set_, typename V>
struct Lookup_Visitor
{
    Dev_Table T;
    const uint64_t* pos_off;
    uint8_t* found;
    V* values;
    uint8_t* fwd;
    uint64_t obase;

    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ void begin_segment(const uint64_t q) { obase = pos_off[q]; }
    __device__ __forceinline__ void end_segment(uint64_t, uint32_t) {}
    __device__ __forceinline__ void lane_begin(const uint64_t q, const bool has) { obase = has ? pos_off[q] : 0; }
    __device__ __forceinline__ void lane_end(uint64_t, bool) {}
    __device__ __forceinline__ void end(uint32_t) {}
    __device__ __forceinline__ void lane_cache(uint4*, uint4*) {}

    __device__ __forceinline__ void visit(const Kmer_Desc& d, const uint32_t)
    {
        const unsigned long long* v = nullptr;
        unsigned long long w = 0;
        if(d.valid)
            v = find_chain<set_, false>(T, d.key, d.h, d.c, w);
        if(!d.in)
            return;
        const uint64_t o = obase + d.pos;
        found[o] = d.valid ? (v ? 1 : 0) : 2;
        if constexpr(!set_)
            if(values)
                values[o] = v ? value_of<V>(w) : V(0);
        if(fwd)
            fwd[o] = d.valid && d.fwd;
    }
};

// Lookups of several batches run as one: each sequence's outputs go to its own batch's arrays, at its positions
// within that batch.
template <bool set_, typename V>
struct Lookup_Batches_Visitor : Lookup_Visitor<set_, V>
{
    const uint32_t* batch_of;   // Sequence -> batch.
    const uint64_t* outs;       // Per batch, 8 words: found, values, fwd at words 4-6 (device addresses, or 0).
    const uint64_t* pos_base;   // Per batch: the merged position of its first k-mer.

    __device__ __forceinline__ void bind(const uint64_t q)
    {
        const uint32_t b = batch_of[q];
        this->found = reinterpret_cast<uint8_t*>(outs[8 * uint64_t(b) + 4]);
        this->values = reinterpret_cast<V*>(outs[8 * uint64_t(b) + 5]);
        this->fwd = reinterpret_cast<uint8_t*>(outs[8 * uint64_t(b) + 6]);
        this->obase = this->pos_off[q] - pos_base[b];
    }
    __device__ __forceinline__ void begin_segment(const uint64_t q) { bind(q); }
    __device__ __forceinline__ void lane_begin(const uint64_t q, const bool has)
    {
        if(has)
            bind(q);
    }
};

// Per-sequence reductions over lookups (capi/Kmer_Table.hpp:134-161): 0 count, 1 masked count, 2 sum. A segment
// belongs to one sequence, so each warp adds its segment's total once.
template <bool set_, typename V, int mode_>
struct Seq_Reduce_Visitor
{
    Dev_Table T;
    unsigned long long* out;
    V m_fwd, m_rev;
    unsigned long long acc;
    unsigned long long total;
    Bucket_Cache bc;
    static constexpr int stage_bytes = 0;

    __device__ __forceinline__ void lane_cache(uint4* lo, uint4* hi) { bc.lo = lo, bc.hi = hi, bc.b = ~0ull; }

    __device__ __forceinline__ void begin() { total = 0; }
    __device__ __forceinline__ void begin(uint8_t*) { total = 0; }
    __device__ __forceinline__ void begin_segment(uint64_t) { acc = 0; }
    __device__ __forceinline__ void visit(const Kmer_Desc& d, const uint32_t)
    {
        if(!d.valid)
            return;
        unsigned long long w = 0;
        if(!find_chain<set_, false>(T, d.key, d.h, d.c, w, bc.lo ? &bc : nullptr))
            return;
        if constexpr(mode_ == 0)
            acc += 1;
        else if constexpr(mode_ == 1)
            acc += (value_of<V>(w) & (d.fwd ? m_fwd : m_rev)) != 0;
        else
            acc += static_cast<unsigned long long>(value_of<V>(w));
    }
    __device__ __forceinline__ void end_segment(const uint64_t q, const uint32_t lane)
    {
        unsigned long long a = acc;
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
        if(lane == 0 && a)
            atomicAdd(out + q, a);
        total += a;
    }
    // One lane, one sequence's segment: its own total.
    __device__ __forceinline__ void lane_begin(uint64_t, bool) { acc = 0; }
    __device__ __forceinline__ void lane_end(const uint64_t q, const bool has)
    {
        if(has && acc)
            atomicAdd(out + q, acc);
    }
    __device__ __forceinline__ void end(uint32_t) {}
};

// The descriptions themselves, for checking the describer.
struct Describe_Visitor
{
    const uint64_t* pos_off;
    uint64_t* key;
    uint64_t* h;
    uint8_t* cs;
    uint8_t* fwd;
    uint8_t* valid;
    bool by_out;    // Outputs at d.out (the lane kernel) rather than pos_off[q] + pos.
    static constexpr int stage_bytes = 0;

    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ void begin(uint8_t*) {}
    __device__ __forceinline__ void begin_segment(uint64_t) {}
    __device__ __forceinline__ void end_segment(uint64_t, uint32_t) {}
    __device__ __forceinline__ void lane_begin(uint64_t, bool) {}
    __device__ __forceinline__ void lane_end(uint64_t, bool) {}
    __device__ __forceinline__ void lane_cache(uint4*, uint4*) {}
    __device__ __forceinline__ void end(uint32_t) {}
    __device__ __forceinline__ void visit(const Kmer_Desc& d, const uint32_t)
    {
        if(!d.in)
            return;
        const uint64_t o = by_out ? d.out : pos_off[d.q] + d.pos;
        key[o] = d.valid ? d.key : 0, h[o] = d.valid ? d.h : 0, cs[o] = d.valid ? d.c : 0;
        fwd[o] = d.valid && d.fwd, valid[o] = d.valid;
    }
};

}
