// The table-wide kernels: resize (rehash into a doubled table), overflow growth, iteration (for_each), reductions,
// histograms, placement statistics, single-k-mer lookups, and the device-side batch preparation.
#pragma once

#include "device_table.cuh"
#include "device_stream.cuh"

namespace kache_b200
{

// Inserts one key with its value, known absent (every key of a table is distinct), into `T`. Returns INSERTED or
// OV_FULL. No other thread inserts the same key, so none waits for the value: no fence before publishing.
template <bool set_>
__device__ __forceinline__ uint32_t place_key(const Dev_Table& T, const uint64_t key, const uint64_t h, const unsigned long long val)
{
    Landing L{};
    const uint32_t r = upsert_chain<set_>(T, key, h, checksum_of(key), L);
    if(r == INSERTED)
    {
        if constexpr(!set_)
            *L.val = val;
        publish(L, false);
        if(!L.cs)
            atomicAdd(T.ov_count, 1ull);
    }
    return r;
}

// Resize, second phase: the old slots marked in `marks` (keys not at their primary bucket, and the overflow table's
// slots) go through the insertion chain of the new table. A warp takes 32 words of marks (1024 slots), lists their set
// bits in shared memory, and then works through the list a slot per lane, so that lanes stay busy however sparse the
// marks are. Keys that find the new overflow table full set their bit in `retry_out`.
template <int k, int l, bool set_>
__global__ void __launch_bounds__(256) rest_kernel(const Dev_Table from, const Dev_Table to, const unsigned int* marks, const uint64_t total,
                                                   unsigned int* retry_out, unsigned int* retried)
{
    __shared__ uint16_t list_all[8][1024];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint16_t* list = list_all[wid];
    const uint64_t main_slots = from.cap * B, words = (total + 31) / 32;
    const uint64_t warps = uint64_t(gridDim.x) * 8;
    for(uint64_t wb = uint64_t(blockIdx.x) * 8 + wid; wb * 32 < words; wb += warps)
    {
        const uint64_t wi = wb * 32 + lane;
        uint32_t word = wi < words ? marks[wi] : 0u;
        if(wi * 32 + 32 > total && wi < words)
            word &= (total - wi * 32) >= 32 ? ~0u : ((1u << (total - wi * 32)) - 1);
        const uint32_t cnt = __popc(word);
        uint32_t pre = cnt;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, pre, o);
            if(lane >= static_cast<uint32_t>(o))
                pre += y;
        }
        const uint32_t n = __shfl_sync(0xFFFFFFFFu, pre, 31);
        pre -= cnt;
        for(uint32_t w = word, i = pre; w; w &= w - 1, ++i)
            list[i] = static_cast<uint16_t>(lane * 32 + __ffs(w) - 1);
        __syncwarp();
        for(uint32_t r = lane; r < n; r += 32)
        {
            const uint64_t s = wb * 1024 + list[r];
            unsigned long long key_st, val = 0;
            if(s < main_slots)
            {
                key_st = from.slots[s * slot_words<set_>()];
                if constexpr(!set_)
                    val = from.slots[s * 2 + 1];
            }
            else
            {
                const uint64_t i = s - main_slots;
                key_st = from.ov[4 * i];
                val = from.ov[4 * i + 1];
            }
            if(key_st == 0)
                continue;
            const uint64_t key = ~key_st;
            if(place_key<set_>(to, key, minimizer_hash<k, l>(key), val) == OV_FULL)
            {
                atomicOr(retry_out + (s >> 5), 1u << (s & 31));
                *retried = 1;
            }
        }
        __syncwarp();
    }
}

// Resize, first phase (include/Streaming_Kmer_Hash_Table.hpp:1494-1570, out of place): a warp per old bucket b.
// The keys whose primary bucket is b move to their primary bucket in the new table, one of the 2^d buckets
// [b * 2^d, (b + 1) * 2^d) when the capacity grows 2^d-fold, since bucket_of is monotone in the capacity; the warp
// writes each of those buckets whole (checksums, keys, values, a cleared spill filter), so the new arrays need no
// clearing. Keys held in b as a secondary bucket get their bit set in `rest`, for the second phase (rest_kernel).
template <int k, int l, bool set_>
__global__ void __launch_bounds__(256) split_kernel(const Dev_Table from, const Dev_Table to, const uint32_t d, unsigned int* rest)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x / 32);
    for(uint64_t b = uint64_t(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5); b < from.cap; b += warps)
    {
        const uint64_t s = b * B + lane;
        const uint8_t c = from.cs[s];
        unsigned long long key_st = 0, val = 0;
        uint32_t dest = 0xFFFFFFFFu;
        if(c)
        {
            key_st = from.slots[s * slot_words<set_>()];
            if constexpr(!set_)
                val = from.slots[s * 2 + 1];
            const uint64_t h = minimizer_hash<k, l>(~key_st);
            if(bucket_of(h, from.cap) == b)
                dest = static_cast<uint32_t>(bucket_of(h, to.cap) - (b << d));
        }
        const uint32_t other = __ballot_sync(0xFFFFFFFFu, c != 0 && dest == 0xFFFFFFFFu);
        if(lane == 0 && other)
            rest[s >> 5] = other;   // s >> 5 == b: one word per old bucket.
        for(uint32_t t = 0; t < (1u << d); ++t)
        {
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, dest == t);
            const uint64_t nb = (b << d) + t;
            // Lane j writes slot j of the new bucket: the rank-j key moving there, or an empty slot.
            const uint32_t n = __popc(m);
            const uint32_t src = lane < n ? __fns(m, 0, static_cast<int>(lane) + 1) : 0;
            const unsigned long long k_j = __shfl_sync(0xFFFFFFFFu, key_st, src);
            const unsigned long long v_j = __shfl_sync(0xFFFFFFFFu, val, src);
            const uint32_t c_j = __shfl_sync(0xFFFFFFFFu, static_cast<uint32_t>(c), src);
            const uint64_t ns = nb * B + lane;
            to.slots[ns * slot_words<set_>()] = lane < n ? k_j : 0ull;
            if constexpr(!set_)
                to.slots[ns * 2 + 1] = lane < n ? v_j : 0ull;
            to.cs[ns] = lane < n ? static_cast<uint8_t>(c_j) : 0;
            if(lane < 8)
                to.spill[nb * 8 + lane] = 0;
        }
    }
}

// Doubles the overflow table: re-inserts its keys into `to`'s overflow table, which has nothing else.
static __global__ void __launch_bounds__(256) ov_move_kernel(const unsigned long long* from, const uint64_t from_slots, const Dev_Table to)
{
    for(uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < from_slots; i += uint64_t(gridDim.x) * blockDim.x)
    {
        const unsigned long long key_st = from[4 * i];
        if(key_st == 0)
            continue;
        // The target has twice the slots, so a free one lies within its capacity.
        uint64_t j = ov_hash(key_st) & to.ov_mask;
        for(uint64_t t = 0; t <= to.ov_mask; ++t, j = (j + 1) & to.ov_mask)
            if(atomicCAS(to.ov + 4 * j, 0ull, key_st) == 0ull)
            {
                to.ov[4 * j + 1] = from[4 * i + 1];
                to.ov[4 * j + 2] = 1;
                break;
            }
    }
}

// Collects the keys (as their 2-bit encodings) and values of buckets [b_b, b_e) and overflow slots [o_b, o_e), in
// no particular order (include/Streaming_Kmer_Hash_Table.hpp:2705-2725): a warp claims its output range with one
// atomic.
template <bool set_>
__global__ void __launch_bounds__(256) collect_kernel(const Dev_Table T, const uint64_t b_b, const uint64_t b_e, const uint64_t o_b, const uint64_t o_e,
                                                      uint64_t* keys, uint64_t* vals, unsigned long long* count)
{
    const uint64_t n_main = (b_e - b_b) * B, total = n_main + (o_e - o_b);
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for(uint64_t s0 = uint64_t(blockIdx.x) * blockDim.x; s0 < total; s0 += stride)
    {
        const uint64_t s = s0 + threadIdx.x;
        bool have = false;
        unsigned long long key_st = 0, val = 0;
        if(s < n_main)
        {
            const uint64_t slot = b_b * B + s;
            if(T.cs[slot])
            {
                have = true;
                key_st = T.slots[slot * slot_words<set_>()];
                if constexpr(!set_)
                    val = T.slots[slot * 2 + 1];
            }
        }
        else if(s < total)
        {
            const uint64_t i = o_b + (s - n_main);
            key_st = T.ov[4 * i];
            if(key_st)
                have = true, val = T.ov[4 * i + 1];
        }
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, have);
        unsigned long long base = 0;
        if(lane == 0 && m)
            base = atomicAdd(count, static_cast<unsigned long long>(__popc(m)));
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if(have)
        {
            const uint64_t o = base + __popc(m & ((1u << lane) - 1));
            keys[o] = ~key_st;
            if(vals)
                vals[o] = val;
        }
    }
}

// Reductions of the C interface over all keys (capi/Kmer_Table.hpp:203-230): 0 keys with v & m nonzero (all keys
// in a set), 1 popcount of v & m, 2 sum of v & m; and 3, the histogram of values in [1, max] (counter/
// Kmer_Set_Counter.cpp:96-119), into `hist`.
template <bool set_, typename V>
__global__ void __launch_bounds__(256) reduce_kernel(const Dev_Table T, const uint32_t what, const uint64_t mask, unsigned long long* out, const uint64_t hmax, unsigned long long* hist)
{
    const uint64_t n_main = T.cap * B, total = n_main + T.ov_mask + 1;
    unsigned long long acc = 0;
    for(uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < total; s += uint64_t(gridDim.x) * blockDim.x)
    {
        bool have;
        unsigned long long raw = 0;
        if(s < n_main)
        {
            have = T.cs[s] != 0;
            if constexpr(!set_)
                if(have)
                    raw = T.slots[s * 2 + 1];
        }
        else
        {
            const uint64_t i = s - n_main;
            have = T.ov[4 * i] != 0;
            if(have)
                raw = T.ov[4 * i + 1];
        }
        if(!have)
            continue;
        const uint64_t v = static_cast<uint64_t>(static_cast<V>(raw));
        if(what == 3)
        {
            if(v >= 1 && v <= hmax)
                atomicAdd(hist + v, 1ull);
            continue;
        }
        const uint64_t x = v & mask;
        if(set_)
            acc += 1;
        else if(what == 0)
            acc += x != 0;
        else if(what == 1)
            acc += __popcll(x);
        else
            acc += x;
    }
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if((threadIdx.x & 31) == 0 && acc)
        atomicAdd(out, acc);
}

// Placement statistics (include/Streaming_Kmer_Hash_Table.hpp:1108-1120,2729-2752): keys in their primary bucket
// and keys in another, from recomputed minimizer hashes.
template <int k, int l, bool set_>
__global__ void __launch_bounds__(256) distribution_kernel(const Dev_Table T, unsigned long long* prim_sec)
{
    const uint64_t n_main = T.cap * B;
    unsigned long long p = 0, s2 = 0;
    for(uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < n_main; s += uint64_t(gridDim.x) * blockDim.x)
    {
        if(!T.cs[s])
            continue;
        const uint64_t key = ~T.slots[s * slot_words<set_>()];
        if(bucket_of(minimizer_hash<k, l>(key), T.cap) == s / B)
            p++;
        else
            s2++;
    }
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        p += __shfl_xor_sync(0xFFFFFFFFu, p, o), s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, o);
    if((threadIdx.x & 31) == 0)
        atomicAdd(prim_sec, p), atomicAdd(prim_sec + 1, s2);
}

// Single k-mer lookups (include/Streaming_Kmer_Hash_Table.hpp:2608-2645) of canonical keys: out[2i] = found,
// out[2i+1] = value.
template <int k, int l, bool set_, typename V>
__global__ void get_kernel(const Dev_Table T, const uint64_t* keys, const uint64_t n, unsigned long long* out)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const uint64_t key = keys[i];
    const unsigned long long* v = find_chain<set_, false>(T, key, minimizer_hash<k, l>(key), checksum_of(key));
    out[2 * i] = v != nullptr;
    out[2 * i + 1] = (v && !set_) ? static_cast<unsigned long long>(read_val<V>(v)) : 0ull;
}

// Device-side batch preparation, for batches already in HBM: per sequence, its positions and segments.
static __global__ void batch_counts_kernel(const uint64_t* off, const uint64_t n, const int k, const uint32_t seg_len, uint64_t* npos, uint64_t* nseg, unsigned int* too_long)
{
    const uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(q >= n)
        return;
    const uint64_t len = off[q + 1] - off[q];
    const uint64_t p = len >= uint64_t(k) ? len - k + 1 : 0;
    npos[q] = p;
    nseg[q] = (p + seg_len - 1) / seg_len;
    if(nseg[q] > max_seg_index + 1)
        atomicOr(too_long, 1u);
}

// The counting and summing of a small device batch's staging in one block of 1024 threads: each thread takes a run
// of sequences; pos_off[0..n] and seg_off[0..n] get the exclusive sums of positions and segments, and out[0..2] the
// positions, the segments and whether a sequence has more segments than a list entry indexes. In place of a counting
// kernel, two scans and their copies; segs_kernel then lists the segments.
constexpr uint32_t small_stage_max = 4096;  // Sequences of a batch summed by one block (at most 4 per thread).

static __global__ void __launch_bounds__(1024) stage_small_kernel(const uint64_t* off, const uint64_t n, const int k, const uint32_t seg_len,
                                                                 uint64_t* pos_off, uint64_t* seg_off, unsigned long long* out)
{
    __shared__ unsigned long long wp[32], ws[32];
    __shared__ unsigned int long_seq;
    const uint32_t t = threadIdx.x, lane = t & 31, wid = t >> 5;
    if(t == 0)
        long_seq = 0;
    const uint64_t per = (n + 1023) / 1024, q0 = min(n, uint64_t(t) * per), q1 = min(n, q0 + per);
    unsigned long long P = 0, S = 0;
    bool too_long = false;
    for(uint64_t q = q0; q < q1; ++q)
    {
        const uint64_t len = off[q + 1] - off[q];
        const uint64_t np = len >= uint64_t(k) ? len - k + 1 : 0, ns = (np + seg_len - 1) / seg_len;
        P += np, S += ns;
        too_long |= ns > max_seg_index + 1;
    }
    // Exclusive prefix sums over the block: within warps by shuffles, then over the warps' totals.
    unsigned long long ip = P, is = S;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1)
    {
        const unsigned long long a = __shfl_up_sync(0xFFFFFFFFu, ip, o), b = __shfl_up_sync(0xFFFFFFFFu, is, o);
        if(lane >= static_cast<uint32_t>(o))
            ip += a, is += b;
    }
    if(lane == 31)
        wp[wid] = ip, ws[wid] = is;
    __syncthreads();
    if(too_long)
        atomicOr(&long_seq, 1u);
    if(wid == 0)
    {
        unsigned long long a = wp[lane], b = ws[lane];
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const unsigned long long x = __shfl_up_sync(0xFFFFFFFFu, a, o), y = __shfl_up_sync(0xFFFFFFFFu, b, o);
            if(lane >= static_cast<uint32_t>(o))
                a += x, b += y;
        }
        wp[lane] = a, ws[lane] = b;
    }
    __syncthreads();
    unsigned long long bp = ip - P + (wid ? wp[wid - 1] : 0), bs = is - S + (wid ? ws[wid - 1] : 0);
    for(uint64_t q = q0; q < q1; ++q)
    {
        const uint64_t len = off[q + 1] - off[q];
        const uint64_t np = len >= uint64_t(k) ? len - k + 1 : 0, ns = (np + seg_len - 1) / seg_len;
        pos_off[q] = bp, seg_off[q] = bs;
        bp += np, bs += ns;
    }
    if(t == 1023)
    {
        pos_off[n] = wp[31], seg_off[n] = ws[31];
        out[0] = wp[31], out[1] = ws[31], out[2] = long_seq;
    }
}

// Lists the segments, one thread per segment: its sequence by binary search in seg_off[0..n] (exclusive sums of
// segments per sequence), so that long sequences' many segments are listed in parallel.
static __global__ void segs_kernel(const uint64_t* seg_off, const uint64_t n, const uint64_t nsegs, uint64_t* segs)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for(uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nsegs; i += stride)
    {
        uint64_t lo = 0, hi = n;      // The last q with seg_off[q] <= i.
        while(hi - lo > 1)
        {
            const uint64_t mid = (lo + hi) / 2;
            if(seg_off[mid] <= i)
                lo = mid;
            else
                hi = mid;
        }
        segs[i] = (lo << 24) | (i - seg_off[lo]);
    }
}



// Several device batches run as one call. desc holds 8 words per batch -- bases, offsets, sequences, first merged
// sequence, out0, out1, out2, 0 -- in batch order. For merged sequence q: its batch, its length (the merged offsets are
// the lengths' sums) and the device address of its first base.
static __global__ void batches_list_kernel(const uint64_t* desc, const uint64_t count, const uint64_t N, uint64_t* lens,
                                           uint64_t* addr, uint32_t* batch_of)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for(uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < N; q += stride)
    {
        uint64_t lo = 0, hi = count;    // The last batch whose first merged sequence is at or before q: never empty.
        while(hi - lo > 1)
        {
            const uint64_t mid = (lo + hi) / 2;
            if(desc[8 * mid + 3] <= q)
                lo = mid;
            else
                hi = mid;
        }
        const uint64_t* off = reinterpret_cast<const uint64_t*>(desc[8 * lo + 1]);
        const uint64_t j = q - desc[8 * lo + 3], a = off[j];
        lens[q] = off[j + 1] - a;
        addr[q] = desc[8 * lo] + a;
        batch_of[q] = static_cast<uint32_t>(lo);
    }
}

// The merged position of each batch's first k-mer.
static __global__ void batches_pos_kernel(const uint64_t* desc, const uint64_t count, const uint64_t* pos_off, uint64_t* pos_base)
{
    const uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(b < count)
        pos_base[b] = pos_off[desc[8 * b + 3]];
}

// Per-batch sums of per-sequence counts: each thread adds a run of consecutive sequences, flushing at batch changes.
static __global__ void batches_sum_kernel(const unsigned long long* per_seq, const uint32_t* batch_of, const uint64_t N,
                                          unsigned long long* per_batch)
{
    const uint64_t threads = uint64_t(gridDim.x) * blockDim.x, t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t per = (N + threads - 1) / threads, q0 = min(N, t * per), q1 = min(N, q0 + per);
    unsigned long long acc = 0;
    uint32_t cur = 0;
    for(uint64_t q = q0; q < q1; ++q)
    {
        const uint32_t b = batch_of[q];
        if(b != cur && acc)
            atomicAdd(per_batch + cur, acc), acc = 0;
        cur = b, acc += per_seq[q];
    }
    if(acc)
        atomicAdd(per_batch + cur, acc);
}

// Per-sequence results of the merged batch copied to each batch's own array (desc word 4).
static __global__ void batches_scatter_kernel(const uint64_t* desc, const unsigned long long* per_seq, const uint32_t* batch_of,
                                              const uint64_t N)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for(uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < N; q += stride)
    {
        const uint64_t b = batch_of[q];
        reinterpret_cast<unsigned long long*>(desc[8 * b + 4])[q - desc[8 * b + 3]] = per_seq[q];
    }
}

// Per-sequence positions found (found flag 1) of a lookup of several batches, read back from each batch's found array
// (desc word 4): a warp per sequence, 4-byte words where aligned, bytes equal to 1 counted by a zero-byte test of the
// word XOR 0x01010101.
static __global__ void batches_hits_kernel(const uint64_t* desc, const uint32_t* batch_of, const uint64_t* pos_off,
                                           const uint64_t* pos_base, const uint64_t N, unsigned long long* per_seq)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x / 32);
    for(uint64_t q = uint64_t(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5); q < N; q += warps)
    {
        const uint32_t b = batch_of[q];
        const uint8_t* f = reinterpret_cast<const uint8_t*>(desc[8 * uint64_t(b) + 4]) + (pos_off[q] - pos_base[b]);
        const uint64_t m = pos_off[q + 1] - pos_off[q];
        const uint64_t lead = (4 - (reinterpret_cast<uintptr_t>(f) & 3)) & 3, head = m < lead ? m : lead;
        const uint64_t nw = (m - head) / 4, tail = head + 4 * nw;
        const uint32_t* w = reinterpret_cast<const uint32_t*>(f + head);
        unsigned long long c = 0;
        if(lane < head)
            c += f[lane] == 1;
#pragma unroll 4
        for(uint64_t i = lane; i < nw; i += 32)
            c += __popc(zero_bytes(w[i] ^ 0x01010101u));
        if(tail + lane < m)
            c += f[tail + lane] == 1;
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
        if(lane == 0)
            per_seq[q] = c;
    }
}

}
