// The C++ template surface of kache-hash's table (include/Streaming_Kmer_Hash_Table.hpp:50-746), on the GPU.
//
// kache_hash::Streaming_Kmer_Hash_Table<k, mt_, T_, l> keeps the reference's members and their meaning: the
// constructor's sizing, register_user and tokens, insert / upsert / upsert_oriented / update / find / count /
// for_each / size / capacity / key_distribution. What changes is where the work runs: value functions `f` are
// device functors, types with a `__device__ T_ operator()(T_) const` (or `(T_, bool) const` for upsert_oriented),
// applied atomically in HBM, possibly more than once per occurrence, so they must have no side effects (as the
// reference's concurrent updates already require, :686-691). Lookup callbacks `g` and iteration callbacks `f` run on
// the host, after the GPU computed every position's result: `g(q, i, r)` or `g(q, i, r, fwd)` per k-mer, in order.
// Include it in a translation unit compiled by nvcc for sm_100a and link libkache_b200.so. `mt_` is accepted and
// ignored: the GPU table is always concurrent.
#pragma once

#include "engine.cuh"

#include <optional>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

namespace kache_hash
{

// A k-mer in its 2-bit encoding, first base most significant, as the reference's Kmer<k>::as_int (include/Kmer.hpp:
// 686-693) gives it to for_each callbacks.
template <uint16_t k>
class Kmer
{
    uint64_t x_ = 0;

public:

    Kmer() = default;
    explicit Kmer(const uint64_t x): x_(x) {}
    uint64_t as_int() const { return x_; }
    bool operator==(const Kmer& o) const { return x_ == o.x_; }
    bool operator<(const Kmer& o) const { return x_ < o.x_; }
    operator std::string() const
    {
        std::string s(k, 'A');
        for(int i = 0; i < k; ++i)
            s[k - 1 - i] = "ACGT"[(x_ >> (2 * i)) & 3];
        return s;
    }
};

template <uint16_t k, bool mt_, typename T_ = void, uint16_t l = 22>
class Streaming_Kmer_Hash_Table
{
    static_assert(k <= 32, "The k-mers need to fit in a machine word.");

public:

    class Token
    {
        friend class Streaming_Kmer_Hash_Table;
        uint16_t id;
        explicit Token(const uint16_t id): id(id) {}

    public:

        Token(): id(0) {}
    };

    static constexpr uint64_t max_user = 128;
    static constexpr double lf_default_ = 0.8;

private:

    static constexpr bool is_set_ = std::is_void_v<T_>;
    static constexpr bool is_map_ = !is_set_;
    typedef typename kache_b200::Val_Of<T_>::type VT;
    typedef std::conditional_t<is_map_, std::optional<VT>, bool> find_ret_t;

    kache_b200::Engine<k, l, T_> E;
    uint16_t users_ = 0;

    // Per-position results of a batch, then the callback per k-mer in order (the reference's lookup callbacks,
    // :2519-2604).
    template <typename G>
    void call_g(const char* const* seqs, const std::size_t* lens, const std::size_t c, const G& g) const
    {
        std::vector<uint64_t> o(c + 1, 0);
        for(std::size_t i = 0; i < c; ++i)
            o[i + 1] = o[i] + (lens[i] >= k ? lens[i] - k + 1 : 0);
        std::vector<uint8_t> found(o[c]), fwd(o[c]);
        std::vector<VT> val(is_map_ ? o[c] : 0);
        auto& e = const_cast<kache_b200::Engine<k, l, T_>&>(E);
        e.lookup(seqs, lens, c, found.data(), is_map_ ? static_cast<void*>(val.data()) : nullptr, fwd.data());
        constexpr bool orient_ = !std::is_invocable_v<const G&, std::size_t, std::size_t, const find_ret_t&> &&
                                 std::is_invocable_v<const G&, std::size_t, std::size_t, const find_ret_t&, bool>;
        for(std::size_t q = 0; q < c; ++q)
            for(uint64_t j = o[q]; j < o[q + 1]; ++j)
            {
                if(found[j] == KACHE_NOT_KMER)
                    continue;
                find_ret_t r;
                if constexpr(is_map_)
                    r = found[j] ? find_ret_t(val[j]) : find_ret_t(std::nullopt);
                else
                    r = found[j] != 0;
                if constexpr(orient_)
                    g(q, j - o[q], r, fwd[j] != 0);
                else
                    g(q, j - o[q], r);
            }
    }

public:

    // Sized as the reference: the fewest buckets for max_sz keys at load lf, rounded up to a power of 2 iff pow2_cap
    // (:771-796). resize_worker_c is accepted and unused.
    explicit Streaming_Kmer_Hash_Table(const std::size_t max_sz = 1 << 22, const uint64_t resize_worker_c = 16, const double lf = lf_default_, const bool pow2_cap = false):
          E(max_sz, lf, pow2_cap)
    {
        (void)resize_worker_c;
    }

    static bool fits(const std::size_t max_sz, const double lf, const bool pow2_cap) { return kache_b200::fits(max_sz, lf, pow2_cap); }

    Streaming_Kmer_Hash_Table(const Streaming_Kmer_Hash_Table&) = delete;
    Streaming_Kmer_Hash_Table& operator=(const Streaming_Kmer_Hash_Table&) = delete;

    auto capacity() const { return E.capacity(); }
    std::size_t bucket_bytes() const { kache_stats s; const_cast<kache_b200::Engine<k, l, T_>&>(E).get_stats(s); return s.bytes; }
    std::size_t size() const { return E.size(); }
    std::size_t overflow_size() const { kache_stats s; const_cast<kache_b200::Engine<k, l, T_>&>(E).get_stats(s); return s.overflow_keys; }

    Token register_user() { return Token(users_++); }

    std::size_t insert(const char* seq, std::size_t len, const Token& token) requires (is_set_) { return insert(&seq, &len, 1, token); }
    std::size_t insert(const char* const* seqs, const std::size_t* lens, const std::size_t c, const Token& token) requires (is_set_)
    {
        return E.upsert(token.id, seqs, lens, c, kache_b200::OP_KEEP, 0, 0);
    }

    template <typename F, typename V = T_>
    std::size_t upsert(const char* seq, std::size_t len, const F& f, const V& val, const Token& token) requires (is_map_) { return upsert(&seq, &len, 1, f, val, token); }

    template <typename F, typename V = T_>
    std::size_t upsert(const char* const* seqs, const std::size_t* lens, const std::size_t c, const F& f, const V& val, const Token& token) requires (is_map_)
    {
        return E.upsert_with(token.id, seqs, lens, c, kache_b200::User_Fn<VT, F>{f, static_cast<VT>(val)});
    }

    template <typename F>
    std::size_t upsert_oriented(const char* const* seqs, const std::size_t* lens, const std::size_t c, const F& f, const Token& token) requires (is_map_)
    {
        return E.upsert_with(token.id, seqs, lens, c, kache_b200::User_Oriented_Fn<VT, F>{f});
    }

    template <typename F> std::size_t update(const char* seq, std::size_t len, const F& f) requires (is_map_) { return update(&seq, &len, 1, f); }

    template <typename F>
    std::size_t update(const char* const* seqs, const std::size_t* lens, const std::size_t c, const F& f) requires (is_map_)
    {
        return E.update_with(seqs, lens, c, kache_b200::User_Fn<VT, F>{f, VT()});
    }

    template <typename G> void find(const char* seq, std::size_t len, const G& g) const
    {
        call_g(&seq, &len, 1, [&](std::size_t, const std::size_t i, const find_ret_t& r){ g(i, r); });
    }

    template <typename G> void find(const char* const* seqs, const std::size_t* lens, const std::size_t c, const G& g) const { call_g(seqs, lens, c, g); }

    find_ret_t find(const char* kmer) const
    {
        uint64_t v = 0;
        const bool hit = const_cast<kache_b200::Engine<k, l, T_>&>(E).get(kmer, v);
        if constexpr(is_map_)
            return hit ? find_ret_t(static_cast<VT>(v)) : find_ret_t(std::nullopt);
        else
            return hit;
    }

    std::size_t count(const char* seq, std::size_t len) const { return count(&seq, &len, 1); }

    std::size_t count(const char* const* seqs, const std::size_t* lens, const std::size_t c) const
    {
        std::vector<uint64_t> cnt(c);
        const_cast<kache_b200::Engine<k, l, T_>&>(E).seq_reduce(seqs, lens, c, 0, 0, 0, cnt.data());
        std::size_t s = 0;
        for(const auto x : cnt)
            s += x;
        return s;
    }

    // f(x) per key of a set, f(x, v) per key and value of a map, over share w_id of w_c (:2705-2725).
    template <typename F> void for_each(const F& f, const std::size_t w_c, const std::size_t w_id) const
    {
        struct Ctx { const F* f; };
        Ctx ctx{&f};
        const_cast<kache_b200::Engine<k, l, T_>&>(E).for_each(static_cast<uint32_t>(w_c), static_cast<uint32_t>(w_id),
            [](void* p, const uint64_t* keys, const void* values, std::size_t n) -> int
            {
                const F& g = *static_cast<Ctx*>(p)->f;
                for(std::size_t i = 0; i < n; ++i)
                    if constexpr(is_set_)
                        g(Kmer<k>(keys[i]));
                    else
                        g(Kmer<k>(keys[i]), static_cast<const VT*>(values)[i]);
                return 0;
            }, &ctx);
    }

    std::tuple<double, double, double> key_distribution() const
    {
        kache_stats s;
        const_cast<kache_b200::Engine<k, l, T_>&>(E).get_stats(s);
        return {s.primary_pct, s.secondary_pct, s.overflow_pct};
    }
};

}
