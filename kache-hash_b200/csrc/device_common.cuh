// Device-side primitives of the B200 streaming k-mer table: hashing, bucket arithmetic, the per-bucket layout.
//
// The arithmetic that decides what a k-mer *is* follows kache-hash bit for bit:
//   - 2-bit codes A0 C1 G2 T3, case-insensitive: ((ch >> 2) ^ (ch >> 1)) & 3      (include/Kmer_Batch.hpp:108)
//   - canonical = min(forward, reverse complement), orientation = key == forward (include/Kmer_Batch.hpp:230-241)
//   - Wang's 64-bit hash, the minimizer hash = least hash of a k-mer's canonical l-mers
//                                                                                 (include/Kmer_Batch.hpp:24-35,204-227)
//   - primary bucket = ((h & 0xFFFFFFFF) * cap) >> 32               (include/Streaming_Kmer_Hash_Table.hpp:1015-1019)
//   - spill-filter index = bits 32..39 of h, 0 mapped to 1           (include/Streaming_Kmer_Hash_Table.hpp:1064-1068)
//   - capacity in buckets = cap_for(n, lf, pow2)                      (include/Streaming_Kmer_Hash_Table.hpp:1004-1011)
// Placement beyond the primary bucket (secondary buckets, the overflow table) is not observable, so it uses its own
// 64-bit mixer where the reference calls XXH3 (include/Streaming_Kmer_Hash_Table.hpp:2112-2115,
// include/Concurrent_Hash_Table.hpp:25-29).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace kache_b200
{

constexpr int B = 32;                  // Slots per bucket: a bucket's 32 checksums fill one 32-byte sector.
constexpr uint64_t max_buckets = (uint64_t(1) << 32) - 1;
constexpr int seg_rows = 16;           // Rows of 32 k-mer positions that one warp describes in a segment.
constexpr int seg_positions = 32 * seg_rows;
constexpr int lane_seg_positions = 64; // Positions of a lane's segment: short, so that a batch has many lanes.
constexpr uint64_t max_seg_index = 0xFFFFFF;   // Segment indexes take 24 bits of a segment list entry.

enum Op : uint32_t { OP_KEEP = 0, OP_ASSIGN = 1, OP_ADD = 2, OP_OR = 3, OP_MIN = 4, OP_MAX = 5, OP_ADD_WRAP = 16 };

// Wang's hash with its shift-and-add steps written as multiplications by constants, modulo 2^64:
// ~x + (x << 21) = x * (2^21 - 1) - 1, x + (x << 3) + (x << 8) = x * 265, x + (x << 2) + (x << 4) = x * 21,
// x + (x << 31) = x * (2^31 + 1). Same value; the multiplies run on the FMA pipe, leaving the integer ALU pipe,
// which the describer saturates, to the shifts and XORs.
__host__ __device__ __forceinline__ uint64_t wang_u64(uint64_t x)
{
    x = x * ((1ull << 21) - 1) - 1;
    x = x ^ (x >> 24);
    x = x * 265;
    x = x ^ (x >> 14);
    x = x * 21;
    x = x ^ (x >> 28);
    x = x * ((1ull << 31) + 1);
    return x;
}

// The key's 8-bit checksum, never 0 (0 marks an empty slot): the top byte of key times an odd constant, as the
// reference's builds without AVX-512 compute it (include/Kmer_Batch.hpp:44-67).
__host__ __device__ __forceinline__ uint8_t checksum_of(const uint64_t key)
{
    const uint8_t c = static_cast<uint8_t>((key * 0x9E3779B97F4A7C15ull) >> 56);
    return c ? c : 1;
}

__device__ __forceinline__ uint64_t min64(const uint64_t a, const uint64_t b) { return a < b ? a : b; }

__host__ __device__ __forceinline__ uint64_t kmer_mask(const int k) { return k == 32 ? ~0ull : (1ull << (2 * k)) - 1; }

__host__ __device__ __forceinline__ uint64_t bucket_of(const uint64_t h, const uint64_t cap)
{
    return ((h & 0xFFFFFFFFull) * cap) >> 32;
}

__host__ __device__ __forceinline__ uint32_t filter_pos(const uint64_t h)
{
    const uint32_t x = static_cast<uint32_t>(h >> 32) & 0xFF;
    return x + (x == 0);
}

// Stafford's 64-bit finaliser (variant 13): the mixer of the unobservable placements.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x ^= x >> 30, x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27, x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

__device__ __forceinline__ uint64_t pick_bucket(const uint64_t x, const uint64_t cap) { return __umul64hi(x, cap); }

// The two secondary buckets of a minimizer hash: one copy of each key, so every inserter of a key scans them in
// this one order, first `p` then `q`.
__device__ __forceinline__ void secondaries(const uint64_t h, const uint64_t cap, uint64_t& p, uint64_t& q)
{
    p = pick_bucket(mix64(h ^ 0x2545F4914F6CDD1Dull), cap);
    q = pick_bucket(mix64(h + 0x9E3779B97F4A7C15ull), cap);
}

__host__ __device__ __forceinline__ uint64_t ov_hash(const uint64_t key) { return mix64(key ^ 0xD6E8FEB86659FD93ull); }

// Reverse complement of a 2k-bit k-mer: complement, reverse the 32 2-bit groups, align.
__device__ __forceinline__ uint64_t revcomp(const uint64_t x, const int k)
{
    uint64_t t = __brevll(~x);
    t = ((t >> 1) & 0x5555555555555555ull) | ((t & 0x5555555555555555ull) << 1);
    return t >> (64 - 2 * k);
}

// The minimizer hash of a canonical key: the least Wang hash of its l-mers' canonical forms
// (include/Kmer_Lanes.hpp:247-274); the l-mer at offset p of the key has its reverse complement at offset k - l - p
// of the key's reverse complement.
template <int k, int l>
__device__ __forceinline__ uint64_t minimizer_hash(const uint64_t key)
{
    constexpr int w = k - l + 1;
    const uint64_t lm = kmer_mask(l);
    const uint64_t r = revcomp(key, k);
    uint64_t h = ~0ull;
#pragma unroll
    for(int p = 0; p < w; ++p)
    {
        const uint64_t f = (key >> (2 * (k - l - p))) & lm;
        const uint64_t b = (r >> (2 * p)) & lm;
        const uint64_t x = wang_u64(f < b ? f : b);
        h = x < h ? x : h;
    }
    return h;
}

// Bit 7 of each byte of the result is set iff that byte of w is zero, exactly (no carries cross bytes).
__device__ __forceinline__ uint32_t zero_bytes(const uint32_t w)
{
    return ~(((w & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | w) & 0x80808080u;
}

// Gathers bits 7, 15, 23, 31 of y into bits 0..3.
__device__ __forceinline__ uint32_t gather4(const uint32_t y)
{
    return (((y >> 7) * 0x00204081u) >> 21) & 0xFu;
}

// The slots of a bucket whose checksum byte (of the 32 bytes a, b) may equal c, as bit 8q + i for byte q of word i,
// that is slot 4i + q (`candidate_slot`): a spread cheaper than slot order. With exact_, exactly the bytes equal to
// c. Without, every byte equal to c and possibly the byte just above one in the same word (the borrow of the
// subtraction reaches it only if it equals c ^ 1): callers verify candidates by their keys.
template <bool exact_>
__device__ __forceinline__ uint32_t candidates32(const uint4 a, const uint4 b, const uint32_t c)
{
    const uint32_t cc = c * 0x01010101u;
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    uint32_t m = 0;
#pragma unroll
    for(int i = 0; i < 8; ++i)
    {
        const uint32_t t = w[i] ^ cc;
        const uint32_t y = exact_ ? zero_bytes(t) : (t - 0x01010101u) & ~t & 0x80808080u;
        m |= y >> (7 - i);
    }
    return m;
}

__device__ __forceinline__ uint32_t candidate_slot(const uint32_t bit) { return 4 * (bit & 7) + (bit >> 3); }

// Bit j of the result is set iff byte j of the 32 bytes (a, b) equals c.
__device__ __forceinline__ uint32_t match32(const uint4 a, const uint4 b, const uint32_t c)
{
    const uint32_t cc = c * 0x01010101u;
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    uint32_t y[8], any = 0;
#pragma unroll
    for(int i = 0; i < 8; ++i)
        y[i] = zero_bytes(w[i] ^ cc), any |= y[i];
    if(!any)
        return 0;
    uint32_t m = 0;
#pragma unroll
    for(int i = 0; i < 8; ++i)
        m |= gather4(y[i]) << (4 * i);
    return m;
}

}
