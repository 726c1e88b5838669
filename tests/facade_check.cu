// Checks of the C++ template surface (kache-hash_b200/csrc/Streaming_Kmer_Hash_Table.cuh) against an exact
// brute-force reference, after the reference's test/check.cpp and test/oriented.cpp: user device functors in upsert,
// upsert_oriented and update; lookups through host callbacks, with and without orientations; counts; single k-mer
// finds in both orientations and with an N; iteration over shares; sizes, inserted totals and capacity growth.
// Built by kache-hash_b200/build.py; run by tests/test_gpu_facade.py. Prints one line, exits 0 iff all agree.
#include "Streaming_Kmer_Hash_Table.cuh"

#include <algorithm>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

using namespace kache_hash;

constexpr uint16_t k = 31, l = 22;

struct Inc
{
    __device__ uint32_t operator()(const uint32_t v) const { return v + 1; }
};

struct Orient_Count
{
    __device__ uint64_t operator()(const uint64_t v, const bool fwd) const { return v + (fwd ? 1 : (uint64_t(1) << 32)); }
};

struct Times3
{
    __device__ uint32_t operator()(const uint32_t v) const { return v * 3 + 1; }
};

static uint64_t rng_state = 88172645463325252ull;
static uint64_t next_rand() { rng_state ^= rng_state << 13, rng_state ^= rng_state >> 7, rng_state ^= rng_state << 17; return rng_state; }

static uint64_t enc(const char* s, bool& ok)
{
    uint64_t x = 0;
    ok = true;
    for(int i = 0; i < k; ++i)
    {
        const char c = static_cast<char>(s[i] | 0x20);
        if(c != 'a' && c != 'c' && c != 'g' && c != 't')
            ok = false;
        x = (x << 2) | static_cast<uint64_t>(((s[i] >> 2) ^ (s[i] >> 1)) & 3);
    }
    return x;
}

static uint64_t rc(uint64_t x)
{
    uint64_t r = 0;
    for(int i = 0; i < k; ++i, x >>= 2)
        r = (r << 2) | (3 - (x & 3));
    return r;
}

int main()
{
    // A genome and reads from it, some reverse-complemented, some with an N.
    std::string g(100000, 'A');
    for(auto& c : g)
        c = "ACGT"[next_rand() & 3];
    std::vector<std::string> reads;
    for(int i = 0; i < 8000; ++i)
    {
        const std::size_t st = next_rand() % (g.size() - 150);
        std::string r = g.substr(st, 150);
        if(i % 2)
        {
            std::string t(r.rbegin(), r.rend());
            for(auto& c : t)
                c = c == 'A' ? 'T' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'A';
            r = t;
        }
        if(i % 11 == 0)
            r[next_rand() % 150] = 'N';
        if(i % 7 == 0)
            for(std::size_t j = 20; j < 60; ++j)
                r[j] |= 0x20;
        reads.push_back(r);
    }

    // The reference's answer: counts per canonical key, and per orientation.
    std::map<uint64_t, uint64_t> cnt, fwd_c, rev_c;
    for(const auto& r : reads)
        for(std::size_t i = 0; i + k <= r.size(); ++i)
        {
            bool ok;
            const uint64_t f = enc(r.data() + i, ok);
            if(!ok)
                continue;
            const uint64_t rv = rc(f), key = std::min(f, rv);
            cnt[key]++;
            (f <= rv ? fwd_c : rev_c)[key]++;
        }

    std::vector<const char*> seqs;
    std::vector<std::size_t> lens;
    for(const auto& r : reads)
        seqs.push_back(r.data()), lens.push_back(r.size());

    int bad = 0;
    // A map of 32-bit counts from a tiny table, which resizes as the reference's does.
    Streaming_Kmer_Hash_Table<k, true, uint32_t, l> M(10);
    auto tok = M.register_user();
    std::size_t ins = 0;
    for(std::size_t i = 0; i < reads.size(); i += 13)
    {
        const std::size_t c = std::min<std::size_t>(13, reads.size() - i);
        ins += M.upsert(seqs.data() + i, lens.data() + i, c, Inc{}, 1u, tok);
    }
    bad += (ins != cnt.size()) + (M.size() != cnt.size()) + (M.capacity() < cnt.size());

    std::size_t calls = 0, wrong = 0;
    M.find(seqs.data(), lens.data(), 200, [&](std::size_t q, std::size_t i, const std::optional<uint32_t>& r)
    {
        calls++;
        bool ok;
        const uint64_t f = enc(reads[q].data() + i, ok);
        const uint64_t key = std::min(f, rc(f));
        wrong += (!ok || !r || *r != cnt[key]);
    });
    std::size_t exp_calls = 0;
    for(std::size_t q = 0; q < 200; ++q)
        for(std::size_t i = 0; i + k <= reads[q].size(); ++i)
        {
            bool ok;
            enc(reads[q].data() + i, ok);
            exp_calls += ok;
        }
    bad += (calls != exp_calls) + (wrong != 0);
    bad += (M.count(seqs.data(), lens.data(), 100) == 0);

    // Single finds in both orientations and with an N.
    std::size_t single_wrong = 0;
    for(std::size_t j = 0; j + k <= 5000; j += 17)
    {
        std::string x = g.substr(j, k);
        bool ok;
        const uint64_t f = enc(x.data(), ok), key = std::min(f, rc(f));
        const auto r = M.find(x.c_str());
        const auto it = cnt.find(key);
        single_wrong += (it == cnt.end()) ? r.has_value() : (!r || *r != it->second);
        x[j % k] = 'N';
        single_wrong += M.find(x.c_str()).has_value();
    }
    bad += single_wrong != 0;

    // Present-only updates with another functor: v -> 3v + 1 once per occurrence; order-free since every occurrence
    // of a key applies the same function... which does not commute with itself only in count, so check one pass of
    // the first read only, whose k-mers occur once in it.
    std::map<uint64_t, uint64_t> after = cnt;
    std::map<uint64_t, int> occ;
    for(std::size_t i = 0; i + k <= reads[1].size(); ++i)
    {
        bool ok;
        const uint64_t f = enc(reads[1].data() + i, ok);
        if(ok)
            occ[std::min(f, rc(f))]++;
    }
    std::size_t present = M.update(seqs[1], lens[1], Times3{});
    std::size_t exp_present = 0;
    for(const auto& [key, n] : occ)
    {
        exp_present += n;
        uint64_t v = after[key];
        for(int t = 0; t < n; ++t)
            v = static_cast<uint32_t>(v * 3 + 1);
        after[key] = v;
    }
    bad += present != exp_present;

    // Iteration over 3 shares: every key once, with its value.
    std::size_t it_c = 0, it_wrong = 0;
    for(std::size_t w = 0; w < 3; ++w)
        M.for_each([&](const Kmer<k>& x, const uint32_t v){ it_c++; it_wrong += (after.count(x.as_int()) == 0 || after[x.as_int()] != v); }, 3, w);
    bad += (it_c != cnt.size()) + (it_wrong != 0);

    // Oriented counts per orientation with a user functor, and oriented lookups.
    Streaming_Kmer_Hash_Table<k, true, uint64_t, l> O(cnt.size());
    auto tok2 = O.register_user();
    const std::size_t ins2 = O.upsert_oriented(seqs.data(), lens.data(), seqs.size(), Orient_Count{}, tok2);
    std::size_t or_wrong = 0;
    O.for_each([&](const Kmer<k>& x, const uint64_t v)
    {
        const uint64_t key = x.as_int();
        or_wrong += ((v & 0xFFFFFFFF) != (fwd_c.count(key) ? fwd_c[key] : 0)) + ((v >> 32) != (rev_c.count(key) ? rev_c[key] : 0));
    }, 1, 0);
    std::size_t fwd_wrong = 0;
    O.find(seqs.data(), lens.data(), 50, [&](std::size_t q, std::size_t i, const std::optional<uint64_t>& r, const bool fw)
    {
        bool ok;
        const uint64_t f = enc(reads[q].data() + i, ok);
        fwd_wrong += (fw != (f <= rc(f))) + !r;
    });
    bad += (ins2 != cnt.size()) + (or_wrong != 0) + (fwd_wrong != 0);

    // A set.
    Streaming_Kmer_Hash_Table<k, true, void, l> S(100);
    auto tok3 = S.register_user();
    const std::size_t ins3 = S.insert(seqs.data(), lens.data(), seqs.size(), tok3);
    std::size_t set_c = 0;
    S.for_each([&](const Kmer<k>& x){ set_c += cnt.count(x.as_int()); }, 1, 0);
    bad += (ins3 != cnt.size()) + (set_c != cnt.size()) + (S.find(g.substr(10, k).c_str()) != true);

    const auto [p, s, o] = M.key_distribution();
    std::printf("facade: keys %zu ins %zu cap %zu calls %zu/%zu wrong %zu single %zu present %zu/%zu iterate %zu/%zu oriented %zu/%zu set %zu placed %.2f/%.2f/%.2f  %s\n",
                M.size(), ins, static_cast<std::size_t>(M.capacity()), calls, exp_calls, wrong, single_wrong, present, exp_present, it_c, it_wrong,
                or_wrong, fwd_wrong, ins3, p, s, o, bad ? "WRONG" : "ok");
    return bad ? 1 : 0;
}
