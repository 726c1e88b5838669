// Checks the lane kernel's autotuner (kache-hash_b200/csrc/seg_tuner.hpp) on the CPU against a synthetic cost per
// candidate: the coordinate search's order (every segment length at the built-in block count from the built-in length
// on, then every block count at the best length), that it then settles on the cheapest candidate it tried, that every
// 64th call retries a neighbour of it in one coordinate, that it follows a cost that changes, and that operations and
// size classes are tuned apart. Prints "ok" and exits 0, or names the first failed check and exits 1.
#include "seg_tuner.hpp"

#include <cstdio>
#include <cstdlib>
#include <vector>

using kache_b200::Seg_Tuner;

namespace
{

int failures = 0;

void expect(const bool ok, const char* what, const int got = -1, const int want = -1)
{
    if(!ok && failures++ == 0)
        std::printf("failed: %s (got %d, want %d)\n", what, got, want);
}

int cand(const int len_i, const int grid_i) { return grid_i * Seg_Tuner::lens + len_i; }

// Milliseconds for a call over `pos` positions with candidate c: cheapest at (len_i, grid_i) = (best_l, best_g).
double cost_ms(const int c, const uint64_t pos, const int best_l, const int best_g)
{
    const int l = c % Seg_Tuner::lens, g = c / Seg_Tuner::lens;
    const double ns_per_pos = 1.0 + 0.25 * std::abs(l - best_l) + 0.5 * std::abs(g - best_g);
    return ns_per_pos * static_cast<double>(pos) * 1e-6;
}

}

int main()
{
    const uint64_t pos = 40000000;      // A size class (2^25 <= pos < 2^26).
    Seg_Tuner t;

    // The first coordinate: the four lengths at the built-in block count, from the built-in length (64) on.
    const int want_first[4] = {cand(2, 0), cand(3, 0), cand(0, 0), cand(1, 0)};
    for(int i = 0; i < 4; ++i)
    {
        const int c = t.pick(0, pos, 64);
        expect(c == want_first[i], "length search order", c, want_first[i]);
        t.record(0, pos, c, cost_ms(c, pos, 3, 2));
    }
    // The second: the other block counts at the best length found (128, index 3).
    for(int g = 1; g < Seg_Tuner::grids; ++g)
    {
        const int c = t.pick(0, pos, 64);
        expect(c == cand(3, g), "block count search order", c, cand(3, g));
        t.record(0, pos, c, cost_ms(c, pos, 3, 2));
    }
    // Then the cheapest tried, (128, 4 blocks), except every 64th call: a neighbour in one coordinate.
    std::vector<int> retries;
    for(int call = 0; call < 300; ++call)
    {
        const int c = t.pick(0, pos, 64);
        if(c != cand(3, 2))
            retries.push_back(c);
        t.record(0, pos, c, cost_ms(c, pos, 3, 2));
    }
    expect(!retries.empty() && retries.size() <= 300 / 64 + 1, "retries only every 64th call", static_cast<int>(retries.size()), 300 / 64);
    for(const int c : retries)
    {
        const int dl = std::abs(c % Seg_Tuner::lens - 3), dg = std::abs(c / Seg_Tuner::lens - 2);
        expect(dl + dg == 1, "a retry is a neighbour of the best in one coordinate", c, cand(3, 2));
    }
    expect(Seg_Tuner::seg_len_of(cand(3, 2)) == 128 && Seg_Tuner::blocks_of(cand(3, 2)) == 4, "candidate decoding");

    // Another operation, and another size class of the same operation, start their own search.
    expect(t.pick(1, pos, 64) == cand(2, 0), "operations tuned apart", t.pick(1, pos, 64), cand(2, 0));
    expect(t.pick(0, pos / 4, 32) == cand(1, 0), "size classes tuned apart", t.pick(0, pos / 4, 32), cand(1, 0));

    // A cost that changes (the table fills): the averages follow it through the retries.
    Seg_Tuner u;
    int last = -1;
    for(int call = 0; call < 2000; ++call)
    {
        const int c = u.pick(2, pos, 64);
        const bool late = call >= 400;
        u.record(2, pos, c, cost_ms(c, pos, late ? 2 : 3, late ? 1 : 2));
        last = c;
    }
    const int settled = u.pick(2, pos, 64);
    expect(settled == cand(2, 1) || last == cand(2, 1), "follows a changed cost to its new best", settled, cand(2, 1));

    if(failures)
        return 1;
    std::printf("ok\n");
    return 0;
}
