// The table in HBM and its lock-free per-k-mer operations.
//
// Layout (structure of arrays, one entry per bucket of B = 32 slots):
//   cs[cap][32]     u8   checksums; 0 = empty. One 32-byte sector per bucket, so one load tests all 32 slots.
//   spill[cap][8]   u32  the 255-bit spill filter of minimizers whose keys left the (full) bucket
//                        (include/Streaming_Kmer_Hash_Table.hpp:91-97,1064-1093). Bit 0 is unused.
//   slots[cap][32]       maps: {u64 ~key, u64 value} (16 B; a key and its value share one sector);
//                        sets: {u64 ~key} (8 B). The key is stored complemented, so zeroed memory is empty: no
//                        canonical k-mer is all T's, whose complement would be 0.
//   ov[ov_cap]           the overflow table: {u64 ~key, u64 value, u64 ready, u64 pad}, linear probing.
//
// Concurrency without locks, in place of the reference's bucket spin locks (include/Streaming_Kmer_Hash_Table.hpp:
// 1125-1212): an insert claims a slot by atomicCAS of its key word from 0, scanning the bucket's slots in order from
// the first empty checksum, so a bucket's claimed keys always form a prefix and every inserter of a key meets any
// earlier claim of it. It then writes the value, fences, and publishes the checksum; a racing inserter of the same key
// that lost the CAS waits (boundedly) for that checksum before applying its update. Every inserter of a key scans the
// same chain -- primary bucket, then secondary p, then q, then the overflow table -- so a key has one copy. A full
// primary bucket gets its spill-filter bit set before any key of its minimizer goes beyond it, which keeps the
// reference's lookup rule: absent past a full primary bucket unless its filter marks the minimizer
// (include/Streaming_Kmer_Hash_Table.hpp:2555-2571).
#pragma once

#include "device_common.cuh"

namespace kache_b200
{

template <typename V> struct Val_Of { typedef V type; static constexpr bool is_set = false; };
template <> struct Val_Of<void> { typedef uint8_t type; static constexpr bool is_set = true; };

struct Dev_Table
{
    uint8_t* cs;
    uint32_t* spill;
    unsigned long long* slots;
    uint64_t cap;           // Buckets.
    unsigned long long* ov; // Overflow slots, 4 words each.
    uint64_t ov_mask;       // Overflow capacity - 1 (a power of 2).
    uint32_t ov_probe;      // Most slots an overflow probe visits.
    unsigned long long* ov_count;   // Keys in the overflow table.
    unsigned int* err;      // Nonzero after a bounded wait gave up.
    uint32_t wait_polls;    // Most polls of a wait for a racing insert's publication.
};

constexpr uint32_t default_wait_polls = 1u << 22;

constexpr uint32_t ERR_WAIT = 1;    // A wait for a racing insert's publication ran out.

template <bool set_> __host__ __device__ constexpr int slot_words() { return set_ ? 1 : 2; }

// Loads that must see other SMs' writes within the same kernel bypass L1.
__device__ __forceinline__ unsigned long long ld_cg(const unsigned long long* p) { return __ldcg(p); }
__device__ __forceinline__ uint4 ld_cg4(const void* p) { return __ldcg(reinterpret_cast<const uint4*>(p)); }
__device__ __forceinline__ uint8_t ld_volatile_u8(const uint8_t* p) { return *reinterpret_cast<const volatile uint8_t*>(p); }

// Reads a stored value as V.
template <typename V>
__device__ __forceinline__ V read_val(const unsigned long long* w)
{
    if constexpr(sizeof(V) == 8)
        return static_cast<V>(*w);
    else
        return static_cast<V>(*reinterpret_cast<const uint32_t*>(w));
}

template <typename V>
__device__ __forceinline__ V read_val_cg(const unsigned long long* w)
{
    if constexpr(sizeof(V) == 8)
        return static_cast<V>(__ldcg(w));
    else
        return static_cast<V>(__ldcg(reinterpret_cast<const uint32_t*>(w)));
}

template <typename V>
__device__ __forceinline__ void write_val(unsigned long long* w, const V v)
{
    if constexpr(sizeof(V) == 8)
        *w = static_cast<unsigned long long>(v);
    else
        *reinterpret_cast<uint32_t*>(w) = static_cast<uint32_t>(v);
}

// Applies `f` to the value at `w` atomically: a compare-and-swap loop on the value's word (the low 32 bits for
// values of up to 4 bytes, whose upper bytes stay 0), as the reference updates values in place
// (include/Streaming_Kmer_Hash_Table.hpp:1239-1253).
template <typename V, typename F>
__device__ __forceinline__ void cas_update(unsigned long long* w, const F& f)
{
    if constexpr(sizeof(V) == 8)
    {
        unsigned long long old = __ldcg(w), assumed;
        do
        {
            assumed = old;
            old = atomicCAS(w, assumed, static_cast<unsigned long long>(f(static_cast<V>(assumed))));
        } while(old != assumed);
    }
    else
    {
        unsigned int* p = reinterpret_cast<unsigned int*>(w);
        unsigned int old = __ldcg(p), assumed;
        do
        {
            assumed = old;
            old = atomicCAS(p, assumed, static_cast<unsigned int>(f(static_cast<V>(assumed))));
        } while(old != assumed);
    }
}

// The closed set of value operations of the C interface (capi/Kmer_Table.hpp:30-43), with a wrapping add for the
// template API's `v + x`: `f(v)` for a present key, `x` for an absent one. Atomic fast paths where one
// instruction does the operation exactly.
template <typename V>
struct Op_Fn
{
    uint32_t op;
    V x;
    V init;

    __device__ __forceinline__ V operator()(const V v) const
    {
        constexpr V mx = static_cast<V>(~V(0));
        switch(op)
        {
        case OP_KEEP: return v;
        case OP_ASSIGN: return x;
        case OP_ADD: return v > static_cast<V>(mx - x) ? mx : static_cast<V>(v + x);
        case OP_OR: return static_cast<V>(v | x);
        case OP_MIN: return v < x ? v : x;
        case OP_ADD_WRAP: return static_cast<V>(v + x);
        default: return v > x ? v : x;
        }
    }

    __device__ __forceinline__ V initial(bool) const { return init; }
    __device__ __forceinline__ bool is_noop() const { return op == OP_KEEP; }

    // Whether every update of a key combines with the others in any order, starting from a zeroed value: then an
    // inserter folds its initial value in atomically (op(0, init) = init for these ops) and nobody waits for it.
    __device__ __forceinline__ bool commutes() const
    {
        return op == OP_KEEP || op == OP_ADD || op == OP_ADD_WRAP || op == OP_OR || op == OP_MAX;
    }

    __device__ __forceinline__ void apply_init(unsigned long long* w, bool) const
    {
        if(op == OP_KEEP)
            write_val<V>(w, init);
        else
            Op_Fn<V>{op, init, init}.apply(w, true);
    }

    __device__ __forceinline__ void apply(unsigned long long* w, bool) const
    {
        if(op == OP_KEEP)
            return;
        constexpr V mx = static_cast<V>(~V(0));
        if constexpr(sizeof(V) == 8)
        {
            switch(op)
            {
            case OP_ADD:
                // Saturating add as an atomic add, then the saturated value wherever an add carried past the maximum:
                // every add that overflows sees it (old > max - x) and stores the maximum after its own add, and an
                // add landing on a value an overflow left small either overflows in turn or is overwritten by that
                // fix-up, so the word ends at min(max, v + sum x) as the serial order would leave it. Nothing reads
                // values while inserts run.
                if(atomicAdd(w, static_cast<unsigned long long>(x)) > static_cast<unsigned long long>(mx - x))
                    atomicExch(w, static_cast<unsigned long long>(mx));
                return;
            case OP_ASSIGN: atomicExch(w, static_cast<unsigned long long>(x)); return;
            case OP_OR: atomicOr(w, static_cast<unsigned long long>(x)); return;
            case OP_MIN: atomicMin(w, static_cast<unsigned long long>(x)); return;
            case OP_MAX: atomicMax(w, static_cast<unsigned long long>(x)); return;
            case OP_ADD_WRAP: atomicAdd(w, static_cast<unsigned long long>(x)); return;
            default: break;
            }
        }
        else
        {
            unsigned int* p = reinterpret_cast<unsigned int*>(w);
            switch(op)
            {
            case OP_ADD:    // As above, on the value's 32-bit word (values of 1 or 2 bytes saturate below its top).
                if(atomicAdd(p, static_cast<unsigned int>(x)) > static_cast<unsigned int>(mx - x))
                    atomicExch(p, static_cast<unsigned int>(mx));
                return;
            case OP_ASSIGN: atomicExch(p, static_cast<unsigned int>(x)); return;
            case OP_OR: atomicOr(p, static_cast<unsigned int>(x)); return;
            case OP_MIN: atomicMin(p, static_cast<unsigned int>(x)); return;
            case OP_MAX: atomicMax(p, static_cast<unsigned int>(x)); return;
            case OP_ADD_WRAP:
                if constexpr(sizeof(V) == 4) { atomicAdd(p, static_cast<unsigned int>(x)); return; }
                break;
            default: break;
            }
        }
        cas_update<V>(w, *this);
    }
};

// The oriented operations (capi/Kmer_Table.hpp:50-61): operand x_fwd for an occurrence as the canonical form,
// x_rev for one as its reverse complement; an absent key gets f(0, fwd) (include/Streaming_Kmer_Hash_Table.hpp:682).
template <typename V>
struct Oriented_Op_Fn
{
    uint32_t op;
    V x_fwd, x_rev;

    __device__ __forceinline__ Op_Fn<V> at(const bool fwd) const { return Op_Fn<V>{op, fwd ? x_fwd : x_rev, V(0)}; }
    __device__ __forceinline__ V initial(const bool fwd) const { return at(fwd)(V(0)); }
    __device__ __forceinline__ bool is_noop() const { return false; }
    __device__ __forceinline__ bool commutes() const { return op == OP_ADD || op == OP_ADD_WRAP || op == OP_OR || op == OP_MAX; }
    __device__ __forceinline__ void apply_init(unsigned long long* w, const bool fwd) const { at(fwd).apply(w, fwd); }
    __device__ __forceinline__ void apply(unsigned long long* w, const bool fwd) const { at(fwd).apply(w, fwd); }
};

// Adapts a user's device functor `f(v)` with the value `val` for absent keys (the C++ template API's upsert).
template <typename V, typename F>
struct User_Fn
{
    F f;
    V val;
    __device__ __forceinline__ V initial(bool) const { return val; }
    __device__ __forceinline__ bool is_noop() const { return false; }
    __device__ __forceinline__ bool commutes() const { return false; }
    __device__ __forceinline__ void apply_init(unsigned long long* w, bool) const { write_val<V>(w, val); }
    __device__ __forceinline__ void apply(unsigned long long* w, bool) const { cas_update<V>(w, f); }
};

// Adapts a user's device functor `f(v, fwd)` (the C++ template API's upsert_oriented): absent keys get f(V(), fwd).
template <typename V, typename F>
struct User_Oriented_Fn
{
    F f;
    __device__ __forceinline__ V initial(const bool fwd) const { return f(V(), fwd); }
    __device__ __forceinline__ bool is_noop() const { return false; }
    __device__ __forceinline__ bool commutes() const { return false; }
    __device__ __forceinline__ void apply_init(unsigned long long* w, const bool fwd) const { write_val<V>(w, f(V(), fwd)); }
    __device__ __forceinline__ void apply(unsigned long long* w, const bool fwd) const
    {
        const F& g = f;
        cas_update<V>(w, [&](const V v){ return g(v, fwd); });
    }
};

// Outcome of one k-mer's upsert chain.
enum Outcome : uint32_t
{
    NONE = 0,
    INSERTED = 1,       // This lane claimed the slot; it still writes the value and publishes.
    FOUND = 2,          // Present and published: apply the update.
    FOUND_PENDING = 3,  // Present, claimed by a racing lane that has yet to publish: wait, then apply.
    OV_FULL = 4         // The overflow table had no room within its probe bound: retry after it grows.
};

template <bool set_>
__device__ __forceinline__ unsigned long long* key_word(const Dev_Table& T, const uint64_t b, const uint32_t j)
{
    return T.slots + (b * B + j) * slot_words<set_>();
}

// A lane's copy, in shared memory, of the checksums of the last primary bucket it probed: consecutive k-mers of a
// read mostly share their minimizer, so their primary bucket, and the copy saves re-reading its sector. The copy may
// miss checksums published since by other lanes. Every probe stays correct with such a copy, only slower: a missed
// candidate of an upsert is met by the claim scan's failed compare-and-swap, whose result is the claimer's key, and
// finds and updates run in kernels without inserts, where nothing changes.
struct Bucket_Cache
{
    uint4* lo;      // Checksums of slots 0..15 and 16..31.
    uint4* hi;
    uint64_t b;     // The bucket copied; ~0 for none.
};

// The checksums of bucket b, from the cache where it holds them, else loaded (and cached).
template <bool cg_>
__device__ __forceinline__ void bucket_cs(const Dev_Table& T, const uint64_t b, Bucket_Cache* bc, uint4& c0, uint4& c1)
{
    if(bc && bc->b == b)
    {
        c0 = *bc->lo, c1 = *bc->hi;
        return;
    }
    const uint8_t* csb = T.cs + b * B;
    c0 = cg_ ? ld_cg4(csb) : *reinterpret_cast<const uint4*>(csb);
    c1 = cg_ ? ld_cg4(csb + 16) : *reinterpret_cast<const uint4*>(csb + 16);
    if(bc)
        *bc->lo = c0, *bc->hi = c1, bc->b = b;
}

// Tries the bucket b for the key: its published candidates, then the claim scan. Returns FOUND, FOUND_PENDING or
// INSERTED with the slot at `j`, or NONE if the bucket is full without the key. With a cache holding b, the cached
// candidates are tried first; if none is the key, the checksums are read afresh (other lanes may have published it
// since), cached, and the probe goes on from them. A slot this lane claims is entered in the cache.
template <bool set_>
__device__ __forceinline__ uint32_t bucket_upsert(const Dev_Table& T, const uint64_t b, const unsigned long long key_st, const uint8_t c, uint32_t& j_out, Bucket_Cache* bc = nullptr)
{
    const uint8_t* csb = T.cs + b * B;
    uint4 c0, c1;
    if(bc && bc->b == b)
    {
        c0 = *bc->lo, c1 = *bc->hi;
        for(uint32_t cand = candidates32<true>(c0, c1, c); cand; cand &= cand - 1)
        {
            const uint32_t j = candidate_slot(__ffs(cand) - 1);
            if(ld_cg(key_word<set_>(T, b, j)) == key_st)
                return j_out = j, FOUND;
        }
    }
    c0 = ld_cg4(csb), c1 = ld_cg4(csb + 16);
    if(bc)
        *bc->lo = c0, *bc->hi = c1, bc->b = b;
    uint32_t cand = candidates32<true>(c0, c1, c);
    while(cand)
    {
        const uint32_t j = candidate_slot(__ffs(cand) - 1);
        cand &= cand - 1;
        if(ld_cg(key_word<set_>(T, b, j)) == key_st)
            return j_out = j, FOUND;
    }
    const uint32_t empty = match32(c0, c1, 0);

    // The claim scan: a compare-and-swap straight away (a slot with an empty checksum is most likely unclaimed), whose
    // result, if it fails, is the racing claimer's key.
    for(uint32_t j = empty ? __ffs(empty) - 1 : B; j < B; ++j)
    {
        unsigned long long* kw = key_word<set_>(T, b, j);
        const unsigned long long cur = atomicCAS(kw, 0ull, key_st);
        if(cur == 0)
        {
            if(bc)
                reinterpret_cast<uint8_t*>(j < 16 ? bc->lo : bc->hi)[j & 15] = c;
            return j_out = j, INSERTED;
        }
        if(cur == key_st)
            return j_out = j, (ld_volatile_u8(csb + j) != 0 ? FOUND : FOUND_PENDING);
    }

    return NONE;
}

// Tries the overflow table. Returns FOUND, FOUND_PENDING or INSERTED with the slot index at `i_out`, or OV_FULL.
__device__ __forceinline__ uint32_t overflow_upsert(const Dev_Table& T, const unsigned long long key_st, uint64_t& i_out)
{
    uint64_t i = ov_hash(key_st) & T.ov_mask;
    for(uint32_t t = 0; t < T.ov_probe; ++t, i = (i + 1) & T.ov_mask)
    {
        unsigned long long* kw = T.ov + 4 * i;
        unsigned long long cur = ld_cg(kw);
        if(cur == 0)
        {
            cur = atomicCAS(kw, 0ull, key_st);
            if(cur == 0)
                return i_out = i, INSERTED;
        }
        if(cur == key_st)
            return i_out = i, (ld_cg(kw + 2) != 0 ? FOUND : FOUND_PENDING);
    }
    return OV_FULL;
}

// Where an upsert chain ended: a value word and the flag that publishes it (a checksum byte, or an overflow slot's
// ready word).
struct Landing
{
    unsigned long long* val;
    uint8_t* cs;            // Non-null in the main table.
    unsigned long long* ready;  // Non-null in the overflow table.
    uint8_t c;
};

// The upsert chain of one k-mer (include/Streaming_Kmer_Hash_Table.hpp:2431-2490, lock-free): primary bucket; if
// full, mark its spill filter, then the secondary buckets in order; then the overflow table.
template <bool set_>
__device__ __forceinline__ uint32_t upsert_chain(const Dev_Table& T, const uint64_t key, const uint64_t h, const uint8_t c, Landing& L, Bucket_Cache* bc = nullptr)
{
    const unsigned long long key_st = ~key;
    uint32_t j;
    const uint64_t b = bucket_of(h, T.cap);
    uint32_t r = bucket_upsert<set_>(T, b, key_st, c, j, bc);
    uint64_t at = b;
    if(r == NONE)
    {
        const uint32_t fp = filter_pos(h);
        uint32_t* sw = T.spill + b * 8 + (fp >> 5);
        const uint32_t bit = 1u << (fp & 31);
        if(!(__ldcg(sw) & bit))
            atomicOr(sw, bit);

        uint64_t p, q;
        secondaries(h, T.cap, p, q);
        r = bucket_upsert<set_>(T, p, key_st, c, j);
        at = p;
        if(r == NONE)
            r = bucket_upsert<set_>(T, q, key_st, c, j), at = q;
    }

    if(r != NONE)
    {
        unsigned long long* kw = key_word<set_>(T, at, j);
        L.val = set_ ? nullptr : kw + 1, L.cs = T.cs + at * B + j, L.ready = nullptr, L.c = c;
        return r;
    }

    uint64_t i;
    r = overflow_upsert(T, key_st, i);
    L.val = T.ov + 4 * i + 1, L.cs = nullptr, L.ready = T.ov + 4 * i + 2, L.c = c;
    return r;
}

// Publishes a claimed slot after its value is written.
__device__ __forceinline__ void publish(const Landing& L, const bool fence)
{
    if(fence)
        __threadfence();
    if(L.cs)
        *reinterpret_cast<volatile uint8_t*>(L.cs) = L.c;
    else
        *reinterpret_cast<volatile unsigned long long*>(L.ready) = 1ull;
}

// Waits, boundedly (`polls` polls), for a racing insert of the same key to publish. Returns false if the wait ran out.
__device__ __forceinline__ bool await_published(const Landing& L, const uint32_t polls)
{
    for(uint32_t t = 0; t < polls; ++t)
    {
        if(L.cs ? ld_volatile_u8(L.cs) != 0 : *reinterpret_cast<const volatile unsigned long long*>(L.ready) != 0)
        {
            __threadfence();
            return true;
        }
        if(t > 64)
            __nanosleep(64);
    }
    return false;
}

// Compares the key of the slot at kw (16-byte aligned for a map) with key_st (a stored, complemented key), keeping its
// value in `val`.
template <bool set_, bool cg_>
__device__ __forceinline__ bool slot_is(const unsigned long long* kw, const unsigned long long key_st, unsigned long long& val)
{
    if constexpr(set_)
        return (cg_ ? ld_cg(kw) : *kw) == key_st;
    else
    {
        const ulonglong2 s = cg_ ? __ldcg(reinterpret_cast<const ulonglong2*>(kw)) : *reinterpret_cast<const ulonglong2*>(kw);
        val = s.y;
        return s.x == key_st;
    }
}

// The candidates of bucket b in `cand` (candidates32's bits), tried in order: the found key's value word (its key word
// in a set), or null.
template <bool set_, bool cg_>
__device__ __forceinline__ unsigned long long* try_candidates(const Dev_Table& T, const uint64_t b, uint32_t cand, const unsigned long long key_st, unsigned long long& val)
{
    while(cand)
    {
        const uint32_t j = candidate_slot(__ffs(cand) - 1);
        cand &= cand - 1;
        unsigned long long* kw = key_word<set_>(T, b, j);
        if(slot_is<set_, cg_>(kw, key_st, val))
            return set_ ? kw : kw + 1;
    }
    return nullptr;
}

// A find past a full primary bucket b (include/Streaming_Kmer_Hash_Table.hpp:2555-2574): absent unless b's spill
// filter marks the minimizer; else the secondary buckets; then the overflow table iff both are full.
template <bool set_, bool cg_>
__device__ __forceinline__ unsigned long long* find_past_primary(const Dev_Table& T, const uint64_t b, const unsigned long long key_st, const uint64_t h, const uint8_t c, unsigned long long& val)
{
    const uint32_t fp = filter_pos(h);
    const uint32_t sw = cg_ ? __ldcg(T.spill + b * 8 + (fp >> 5)) : T.spill[b * 8 + (fp >> 5)];
    if(!((sw >> (fp & 31)) & 1))
        return nullptr;

    uint64_t p, q;
    secondaries(h, T.cap, p, q);
    bool full_p = false, full_q = false;
    for(int t = 0; t < 2; ++t)
    {
        const uint64_t s = t ? q : p;
        uint4 c0, c1;
        bucket_cs<cg_>(T, s, nullptr, c0, c1);
        if(auto* r = try_candidates<set_, cg_>(T, s, candidates32<false>(c0, c1, c), key_st, val))
            return r;
        (t ? full_q : full_p) = (c1.w >> 24) != 0;
    }
    if(!(full_p && full_q))
        return nullptr;

    uint64_t i = ov_hash(key_st) & T.ov_mask;
    for(uint32_t t = 0; t < T.ov_probe; ++t, i = (i + 1) & T.ov_mask)
    {
        unsigned long long* kw = T.ov + 4 * i;
        const ulonglong2 s = cg_ ? __ldcg(reinterpret_cast<const ulonglong2*>(kw)) : *reinterpret_cast<const ulonglong2*>(kw);
        if(s.x == key_st)
            return val = s.y, kw + 1;
        if(s.x == 0)
            return nullptr;
    }
    return nullptr;
}

// Finds a key: primary bucket; absent if it is not full, or if its spill filter does not mark the minimizer; else the
// secondary buckets; then the overflow table iff both are full (include/Streaming_Kmer_Hash_Table.hpp:2548-2574).
// Returns the value word (the key word for a set), or null if absent; a map's value word, read together with its key
// in one 16-byte load, also goes to `val`.
template <bool set_, bool cg_>
__device__ __forceinline__ unsigned long long* find_chain(const Dev_Table& T, const uint64_t key, const uint64_t h, const uint8_t c, unsigned long long& val, Bucket_Cache* bc = nullptr)
{
    const unsigned long long key_st = ~key;
    const uint64_t b = bucket_of(h, T.cap);
    uint4 c0, c1;
    bucket_cs<cg_>(T, b, bc, c0, c1);
    if(auto* r = try_candidates<set_, cg_>(T, b, candidates32<false>(c0, c1, c), key_st, val))
        return r;
    if((c1.w >> 24) == 0)   // Keys fill a bucket's slots in order: full iff its last checksum is set.
        return nullptr;
    return find_past_primary<set_, cg_>(T, b, key_st, h, c, val);
}

template <bool set_, bool cg_>
__device__ __forceinline__ unsigned long long* find_chain(const Dev_Table& T, const uint64_t key, const uint64_t h, const uint8_t c, Bucket_Cache* bc = nullptr)
{
    unsigned long long val;
    return find_chain<set_, cg_>(T, key, h, c, val, bc);
}

// For failure-injection tests: claims a slot of the key's primary bucket for it, as a racing inserter would, and
// leaves it unpublished (its checksum stays 0), so that a later inserter of the key that must see its value first
// waits on it. One thread; *ok is set to 1 if a slot was claimed.
template <int k, int l, bool set_>
__global__ void plant_claim_kernel(const Dev_Table T, const uint64_t key, unsigned long long* ok)
{
    const uint64_t b = bucket_of(minimizer_hash<k, l>(key), T.cap);
    const uint4 c0 = *reinterpret_cast<const uint4*>(T.cs + b * B), c1 = *reinterpret_cast<const uint4*>(T.cs + b * B + 16);
    const uint32_t empty = match32(c0, c1, 0);
    *ok = 0;
    if(!empty)
        return;
    unsigned long long* kw = key_word<set_>(T, b, __ffs(empty) - 1);
    *ok = atomicCAS(kw, 0ull, ~key) == 0ull;
}

// The value of a found key, as read with it.
template <typename V>
__device__ __forceinline__ V value_of(const unsigned long long w)
{
    if constexpr(sizeof(V) == 8)
        return static_cast<V>(w);
    else
        return static_cast<V>(static_cast<uint32_t>(w));
}

}
