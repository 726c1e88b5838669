// Checks Stream_Writer (kache-hash_b200/csrc/host_copy.hpp) on the CPU: runs of random lengths gathered end to end
// from every destination alignment must equal the same gather by memcpy, and no byte outside the destination range
// may change. Prints "ok" and exits 0, or names the first difference and exits 1.
#include "host_copy.hpp"

#include <cstdio>
#include <random>
#include <vector>

using kache_b200::Stream_Writer;

int main()
{
    std::mt19937_64 rng(71);
    std::vector<char> src(1 << 22);
    for(auto& c : src)
        c = static_cast<char>(rng());
    for(int trial = 0; trial < 400; ++trial)
    {
        const size_t runs = rng() % 200;
        const size_t max_len = trial % 4 == 0 ? 9000 : trial % 4 == 1 ? 40 : trial % 4 == 2 ? 160 : 1;
        std::vector<std::pair<size_t, size_t>> rs;
        size_t total = 0;
        for(size_t r = 0; r < runs; ++r)
        {
            const size_t len = rng() % (max_len + 1), at = rng() % (src.size() - len);
            rs.emplace_back(at, len);
            total += len;
        }
        const size_t align = trial % 16, guard = 64;
        std::vector<char> want(total + align + 2 * guard, 'G'), got(total + align + 2 * guard, 'G');
        char* w0 = want.data() + guard + align;
        char* g0 = got.data() + guard + align;
        size_t o = 0;
        for(const auto& [at, len] : rs)
            std::memcpy(w0 + o, src.data() + at, len), o += len;
        Stream_Writer w(g0);
        for(const auto& [at, len] : rs)
            w.put(src.data() + at, len);
        w.finish();
        if(w.written() != total)
        {
            std::printf("trial %d: written %zu of %zu\n", trial, w.written(), total);
            return 1;
        }
        for(size_t i = 0; i < want.size(); ++i)
            if(want[i] != got[i])
            {
                std::printf("trial %d (align %zu, %zu runs, %zu bytes): byte %zd differs\n", trial, align, runs, total,
                            static_cast<ptrdiff_t>(i) - static_cast<ptrdiff_t>(guard + align));
                return 1;
            }
    }
    std::vector<uint64_t> words(1000, 7);
    for(size_t i = 1; i < 999; ++i)
        kache_b200::stream_u64(words.data() + i, i * 0x9E3779B97F4A7C15ull);
    kache_b200::stream_fence();
    for(size_t i = 0; i < 1000; ++i)
        if(words[i] != ((i == 0 || i == 999) ? 7 : i * 0x9E3779B97F4A7C15ull))
        {
            std::printf("stream_u64: word %zu differs\n", i);
            return 1;
        }
    std::printf("ok\n");
    return 0;
}
