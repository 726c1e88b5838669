// Second opinion for the checker, and the timed CPU baseline: a thin C surface over the reference's own
// Streaming_Kmer_Hash_Table (kache-hash include/Streaming_Kmer_Hash_Table.hpp), compiled from the reference's
// headers where they lie (see oracle/Makefile). It is test and benchmark infrastructure only: nothing in the
// product links or loads it.
//
// Batches come in as one buffer of concatenated sequences plus n+1 offsets; each entry point rebuilds the
// `seqs`/`lens` arrays the reference's batch operations take (Streaming_Kmer_Hash_Table.hpp:659,672,682,698,712).

#include "Streaming_Kmer_Hash_Table.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <type_traits>
#include <vector>

using namespace kache_hash;

namespace
{

enum Op : uint32_t { KEEP = 0, ASSIGN = 1, ADD = 2, OR = 3, MIN = 4, MAX = 5, ADD_WRAP = 16 };

struct Batch
{
    std::vector<const char*> seqs;
    std::vector<std::size_t> lens;
    Batch(const char* bases, const uint64_t* off, std::size_t n, std::size_t b = 0, std::size_t e = SIZE_MAX)
    {
        e = std::min(e, n);
        for(std::size_t i = b; i < e; ++i)
            seqs.push_back(bases + off[i]), lens.push_back(off[i + 1] - off[i]);
    }
    std::size_t size() const { return seqs.size(); }
};

// Runs `g(f)` with the value function of the operation `op` and operand `x`, as the reference's C interface
// defines the operations (capi/Kmer_Table.hpp:30-43), plus a wrapping add for the template API's `v + x`.
template <typename V, typename G>
auto with_op(uint32_t op, V x, const G& g)
{
    constexpr V mx = std::numeric_limits<V>::max();
    switch(op)
    {
    case KEEP:     return g([](const V v){ return v; });
    case ASSIGN:   return g([x](V){ return x; });
    case ADD:      return g([x](const V v){ return static_cast<V>(v > mx - x ? mx : v + x); });
    case OR:       return g([x](const V v){ return static_cast<V>(v | x); });
    case MIN:      return g([x](const V v){ return std::min(v, x); });
    case ADD_WRAP: return g([x](const V v){ return static_cast<V>(v + x); });
    default:       return g([x](const V v){ return std::max(v, x); });
    }
}

template <typename V, typename G>
auto with_oriented_op(uint32_t op, V xf, V xr, const G& g)
{
    constexpr V mx = std::numeric_limits<V>::max();
    switch(op)
    {
    case ASSIGN:   return g([xf, xr](V, const bool f){ return f ? xf : xr; });
    case ADD:      return g([xf, xr](const V v, const bool f){ const V x = f ? xf : xr; return static_cast<V>(v > mx - x ? mx : v + x); });
    case OR:       return g([xf, xr](const V v, const bool f){ return static_cast<V>(v | (f ? xf : xr)); });
    case ADD_WRAP: return g([xf, xr](const V v, const bool f){ return static_cast<V>(v + (f ? xf : xr)); });
    default:       return g([xf, xr](const V v, const bool f){ return std::max(v, f ? xf : xr); });
    }
}

struct Table
{
    virtual ~Table() = default;
    virtual uint32_t reg() = 0;
    virtual uint64_t upsert(uint32_t u, const Batch& b, uint32_t op, uint64_t x) = 0;
    virtual uint64_t upsert_oriented(uint32_t u, const Batch& b, uint32_t op, uint64_t xf, uint64_t xr) = 0;
    virtual uint64_t update(const Batch& b, uint32_t op, uint64_t x) = 0;
    virtual void lookup(const Batch& b, const uint64_t* pos_off, uint8_t* found, uint64_t* val, uint8_t* fwd) const = 0;
    virtual uint64_t count(const Batch& b) const = 0;
    virtual int get(const char* kmer, uint64_t* v) const = 0;
    virtual uint64_t size() const = 0;
    virtual uint64_t capacity() const = 0;
    virtual uint64_t overflow_size() const = 0;
    virtual uint64_t dump(uint64_t* keys, uint64_t* vals, std::size_t w_c, std::size_t w_id) const = 0;
};

template <uint16_t k, typename V, uint16_t l>
struct Table_Of final : Table
{
    static constexpr bool is_set = std::is_void_v<V>;
    typedef std::conditional_t<is_set, uint8_t, V> val_t;
    typedef Streaming_Kmer_Hash_Table<k, true, V, l> table_t;

    table_t M;
    std::vector<typename table_t::Token> tok;

    Table_Of(uint64_t n, double lf, bool pow2, unsigned workers): M(n, workers, lf, pow2) {}

    uint32_t reg() override { tok.push_back(M.register_user()); return tok.size() - 1; }

    uint64_t upsert(uint32_t u, const Batch& b, uint32_t op, uint64_t x) override
    {
        if constexpr(is_set)
            return (void)op, (void)x, M.insert(b.seqs.data(), b.lens.data(), b.size(), tok[u]);
        else
            return with_op(op, static_cast<V>(x), [&](const auto& f){ return M.upsert(b.seqs.data(), b.lens.data(), b.size(), f, static_cast<V>(x), tok[u]); });
    }

    uint64_t upsert_oriented(uint32_t u, const Batch& b, uint32_t op, uint64_t xf, uint64_t xr) override
    {
        if constexpr(is_set)
            return (void)u, (void)b, (void)op, (void)xf, (void)xr, 0;
        else
            return with_oriented_op(op, static_cast<V>(xf), static_cast<V>(xr), [&](const auto& f){ return M.upsert_oriented(b.seqs.data(), b.lens.data(), b.size(), f, tok[u]); });
    }

    uint64_t update(const Batch& b, uint32_t op, uint64_t x) override
    {
        if constexpr(is_set)
            return (void)b, (void)op, (void)x, 0;
        else
            return with_op(op, static_cast<V>(x), [&](const auto& f){ return M.update(b.seqs.data(), b.lens.data(), b.size(), f); });
    }

    void lookup(const Batch& b, const uint64_t* o, uint8_t* found, uint64_t* val, uint8_t* fwd) const override
    {
        M.find(b.seqs.data(), b.lens.data(), b.size(), [&](const std::size_t q, const std::size_t i, const auto& r, const bool f)
        {
            const auto j = o[q] + i;
            found[j] = static_cast<bool>(r) ? 1 : 0;
            if constexpr(!is_set)
                if(val)
                    val[j] = r ? static_cast<uint64_t>(*r) : 0;
            if(fwd)
                fwd[j] = f;
        });
    }

    uint64_t count(const Batch& b) const override { return M.count(b.seqs.data(), b.lens.data(), b.size()); }

    int get(const char* kmer, uint64_t* v) const override
    {
        const auto r = M.find(kmer);
        if constexpr(is_set)
            return *v = 0, r ? 1 : 0;
        else
            return *v = r.value_or(0), r.has_value() ? 1 : 0;
    }

    uint64_t size() const override { return M.size(); }
    uint64_t capacity() const override { return M.capacity(); }
    uint64_t overflow_size() const override { return M.overflow_size(); }

    uint64_t dump(uint64_t* keys, uint64_t* vals, std::size_t w_c, std::size_t w_id) const override
    {
        uint64_t c = 0;
        if constexpr(is_set)
            M.for_each([&](const Kmer<k>& x){ keys[c] = x.as_int(); if(vals) vals[c] = 0; c++; }, w_c, w_id);
        else
            M.for_each([&](const Kmer<k>& x, const V v){ keys[c] = x.as_int(); if(vals) vals[c] = v; c++; }, w_c, w_id);
        return c;
    }
};

Table* make(uint32_t kind, uint64_t n, double lf, bool pow2, unsigned workers)
{
    switch(kind)
    {
    case 0:  return new Table_Of<31, uint64_t, 22>(n, lf, pow2, workers);
    case 1:  return new Table_Of<31, uint32_t, 22>(n, lf, pow2, workers);
    case 2:  return new Table_Of<31, uint16_t, 22>(n, lf, pow2, workers);
    case 3:  return new Table_Of<31, uint8_t, 22>(n, lf, pow2, workers);
    case 4:  return new Table_Of<31, void, 22>(n, lf, pow2, workers);
    case 5:  return new Table_Of<27, uint8_t, 16>(n, lf, pow2, workers);
    case 6:  return new Table_Of<32, void, 20>(n, lf, pow2, workers);
    case 7:  return new Table_Of<27, uint64_t, 16>(n, lf, pow2, workers);
    default: return nullptr;
    }
}

double now_s() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

}


// The reference's batch describer (include/Kmer_Batch.hpp) over a sequence split into ACGT stretches
// (include/DNA_Utility.hpp:199-224), per position: canonical key, minimizer hash, checksum, orientation, validity;
// and the lane describer's minimizer hashes recomputed from the keys (include/Kmer_Lanes.hpp:247-274).
template <uint16_t k, uint16_t l>
uint64_t describe_with(const char* s, uint64_t len, uint64_t* key, uint64_t* h, uint8_t* cs, uint8_t* fwd, uint8_t* valid, uint64_t* h_lanes)
{
    if(len < k)
        return 0;
    const uint64_t n = len - k + 1;
    std::fill(key, key + n, 0), std::fill(h, h + n, 0), std::fill(cs, cs + n, 0), std::fill(fwd, fwd + n, 0), std::fill(valid, valid + n, 0);
    std::fill(h_lanes, h_lanes + n, 0);
    typedef Kmer_Batch<k, l> batch_t;
    batch_t kb;
    typename batch_t::Oriented_Chunk ch;
    for(uint64_t st = 0; st + k <= len; )
    {
        const uint64_t e = st + DNA_Utility::acgt_prefix(s + st, len - st);
        if(e - st >= k)
        {
            kb.reset(s + st, e - st - (k - 1));
            uint64_t at = st;
            while(kb.next(ch))
            {
                for(std::size_t i = 0; i < ch.n; ++i)
                    key[at + i] = ch.key[i], h[at + i] = ch.h[i], cs[at + i] = ch.c[i], fwd[at + i] = ch.o[i], valid[at + i] = 1;
                Kmer_Lanes<k, l>::minimizer_hashes(ch.key, ch.n, h_lanes + at);
                at += ch.n;
            }
        }
        st = e + 1;
    }
    return n;
}

extern "C"
{

// Table kinds: 0 <31,u64,22>, 1 <31,u32,22>, 2 <31,u16,22>, 3 <31,u8,22>, 4 <31,void,22>, 5 <27,u8,16>,
// 6 <32,void,20>, 7 <27,u64,16>; all concurrent (`mt_ = true`).
void* ref_new(uint32_t kind, uint64_t n, double lf, int pow2, unsigned workers) { return make(kind, n, lf, pow2 != 0, workers); }
void ref_free(void* t) { delete static_cast<Table*>(t); }
uint32_t ref_register(void* t) { return static_cast<Table*>(t)->reg(); }

uint64_t ref_upsert(void* t, uint32_t u, const char* bases, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x)
{
    return static_cast<Table*>(t)->upsert(u, Batch(bases, off, n), op, x);
}

uint64_t ref_upsert_oriented(void* t, uint32_t u, const char* bases, const uint64_t* off, uint64_t n, uint32_t op, uint64_t xf, uint64_t xr)
{
    return static_cast<Table*>(t)->upsert_oriented(u, Batch(bases, off, n), op, xf, xr);
}

uint64_t ref_update(void* t, const char* bases, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x)
{
    return static_cast<Table*>(t)->update(Batch(bases, off, n), op, x);
}

// Per-position results at `pos_off[q] + i`; `pos_off` has the positions of the sequences before each.
void ref_lookup(void* t, const char* bases, const uint64_t* off, uint64_t n, const uint64_t* pos_off, uint8_t* found, uint64_t* val, uint8_t* fwd)
{
    static_cast<Table*>(t)->lookup(Batch(bases, off, n), pos_off, found, val, fwd);
}

uint64_t ref_count(void* t, const char* bases, const uint64_t* off, uint64_t n) { return static_cast<Table*>(t)->count(Batch(bases, off, n)); }
int ref_get(void* t, const char* kmer, uint64_t* v) { return static_cast<Table*>(t)->get(kmer, v); }
uint64_t ref_size(void* t) { return static_cast<Table*>(t)->size(); }
uint64_t ref_capacity(void* t) { return static_cast<Table*>(t)->capacity(); }
uint64_t ref_overflow_size(void* t) { return static_cast<Table*>(t)->overflow_size(); }
uint64_t ref_dump(void* t, uint64_t* keys, uint64_t* vals) { return static_cast<Table*>(t)->dump(keys, vals, 1, 0); }

uint64_t ref_describe(uint32_t k, const char* s, uint64_t len, uint64_t* key, uint64_t* h, uint8_t* cs, uint8_t* fwd, uint8_t* valid, uint64_t* h_lanes)
{
    switch(k)
    {
    case 31: return describe_with<31, 22>(s, len, key, h, cs, fwd, valid, h_lanes);
    case 27: return describe_with<27, 16>(s, len, key, h, cs, fwd, valid, h_lanes);
    case 32: return describe_with<32, 20>(s, len, key, h, cs, fwd, valid, h_lanes);
    default: return 0;
    }
}

// The CPU baseline's drivers, as the reference's benchmark drives its table (benchmark/measure.cpp:45-140,
// benchmark/harness.hpp:268-303): batches of `batch` sequences handed to `threads` users round-robin. Return
// the wall seconds; put the sum of the calls' results at `*out`.
double ref_bench_upsert(void* tv, const char* bases, const uint64_t* off, uint64_t n, uint32_t batch, uint32_t threads, uint32_t op, uint64_t x, uint64_t* out)
{
    auto* t = static_cast<Table*>(tv);
    std::vector<uint32_t> users(threads);
    for(auto& u : users)
        u = t->reg();
    std::atomic<uint64_t> next{0}, total{0};
    const double t0 = now_s();
    std::vector<std::thread> W;
    for(uint32_t w = 0; w < threads; ++w)
        W.emplace_back([&, w]()
        {
            uint64_t c = 0;
            for(uint64_t b; (b = next++) * batch < n; )
                c += t->upsert(users[w], Batch(bases, off, n, b * batch, (b + 1) * batch), op, x);
            total += c;
        });
    for(auto& w : W)
        w.join();
    *out = total;
    return now_s() - t0;
}

// As ref_bench_upsert, for upsert_oriented (op, x_fwd, x_rev) and for present-only updates (op, x).
double ref_bench_upsert_oriented(void* tv, const char* bases, const uint64_t* off, uint64_t n, uint32_t batch, uint32_t threads, uint32_t op, uint64_t xf, uint64_t xr, uint64_t* out)
{
    auto* t = static_cast<Table*>(tv);
    std::vector<uint32_t> users(threads);
    for(auto& u : users)
        u = t->reg();
    std::atomic<uint64_t> next{0}, total{0};
    const double t0 = now_s();
    std::vector<std::thread> W;
    for(uint32_t w = 0; w < threads; ++w)
        W.emplace_back([&, w]()
        {
            uint64_t c = 0;
            for(uint64_t b; (b = next++) * batch < n; )
                c += t->upsert_oriented(users[w], Batch(bases, off, n, b * batch, (b + 1) * batch), op, xf, xr);
            total += c;
        });
    for(auto& w : W)
        w.join();
    *out = total;
    return now_s() - t0;
}

double ref_bench_update(void* tv, const char* bases, const uint64_t* off, uint64_t n, uint32_t batch, uint32_t threads, uint32_t op, uint64_t x, uint64_t* out)
{
    auto* t = static_cast<Table*>(tv);
    std::atomic<uint64_t> next{0}, total{0};
    const double t0 = now_s();
    std::vector<std::thread> W;
    for(uint32_t w = 0; w < threads; ++w)
        W.emplace_back([&]()
        {
            uint64_t c = 0;
            for(uint64_t b; (b = next++) * batch < n; )
                c += t->update(Batch(bases, off, n, b * batch, (b + 1) * batch), op, x);
            total += c;
        });
    for(auto& w : W)
        w.join();
    *out = total;
    return now_s() - t0;
}

double ref_bench_count(void* tv, const char* bases, const uint64_t* off, uint64_t n, uint32_t batch, uint32_t threads, uint64_t* out)
{
    auto* t = static_cast<Table*>(tv);
    std::atomic<uint64_t> next{0}, total{0};
    const double t0 = now_s();
    std::vector<std::thread> W;
    for(uint32_t w = 0; w < threads; ++w)
        W.emplace_back([&]()
        {
            uint64_t c = 0;
            for(uint64_t b; (b = next++) * batch < n; )
                c += t->count(Batch(bases, off, n, b * batch, (b + 1) * batch));
            total += c;
        });
    for(auto& w : W)
        w.join();
    *out = total;
    return now_s() - t0;
}


// Per-position finds (found flag and value at pos_off[q] + i), in batches of `batch` sequences over `threads`
// threads; returns the wall seconds.
double ref_bench_lookup(void* tv, const char* bases, const uint64_t* off, uint64_t n, const uint64_t* pos_off, uint32_t batch, uint32_t threads, uint8_t* found, uint64_t* val)
{
    auto* t = static_cast<Table*>(tv);
    std::atomic<uint64_t> next{0};
    const double t0 = now_s();
    std::vector<std::thread> W;
    for(uint32_t w = 0; w < threads; ++w)
        W.emplace_back([&]()
        {
            for(uint64_t b; (b = next++) * batch < n; )
                t->lookup(Batch(bases, off, n, b * batch, (b + 1) * batch), pos_off + b * batch, found, val, nullptr);
        });
    for(auto& w : W)
        w.join();
    return now_s() - t0;
}

}
