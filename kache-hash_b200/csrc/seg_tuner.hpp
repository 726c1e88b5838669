// The lane kernel's online autotuner: host logic only, kept apart from the CUDA code so that it can be checked on
// the CPU (tests/tuner_check.cpp).
#pragma once

#include <cstdint>

namespace kache_b200
{

// Picks the lane kernel's launch shape per operation (upsert, update, per-sequence reduction) and batch size class (the
// log2 of its positions), online, over two dimensions:
//   - the segment length, positions per lane: how many lanes a batch has and how much of each lane's rolling is
//     warm-up (k - 1 bases per segment);
//   - the blocks launched per SM, which take segments from the work counter: how many of the kernel's warps are
//     resident at once against how long the last ones run alone.
// Candidate c is segment length len[c % 4] at blocks[c / 4] per SM. The first calls of a class search coordinate by
// coordinate: every segment length at the built-in block count, then every block count at the best length so far.
// Later calls take the fastest per position (a moving average of the event-timed kernel time), and every 64th call
// retries a neighbour of the best so the averages follow the table as it fills.
class Seg_Tuner
{
public:
    static constexpr int lens = 4, grids = 3, cands = lens * grids;
    static constexpr uint32_t len[lens] = {16, 32, 64, 128};
    // Per SM; the first is the built-in count. Not two: the lane kernels are latency-bound and need their resident
    // warps (the config-1 upsert took 1.85-1.89 ms at three resident blocks against 1.62-1.67 at four), so two would
    // only cost each size class a slow exploring call.
    static constexpr uint32_t blocks[grids] = {16, 8, 4};

    static uint32_t seg_len_of(const int c) { return len[c % lens]; }
    static uint32_t blocks_of(const int c) { return blocks[c / lens]; }

    // The candidate for a call of `kind` over `pos` positions; `dflt` is the built-in segment length.
    int pick(const int kind, const uint64_t pos, const uint32_t dflt)
    {
        Slot& s = slot(kind, pos);
        int d = 0;
        while(d + 1 < lens && len[d] < dflt)
            d++;
        for(int i = 0; i < lens; ++i)       // First coordinate: segment lengths at the built-in block count.
        {
            const int c = (d + i) % lens;
            if(s.tries[c] == 0)
                return c;
        }
        int best_len = 0;
        for(int c = 1; c < lens; ++c)
            if(s.ns_per_pos[c] < s.ns_per_pos[best_len])
                best_len = c;
        for(int g = 1; g < grids; ++g)      // Second: block counts at the best length.
            if(s.tries[g * lens + best_len] == 0)
                return g * lens + best_len;
        int best = best_len;
        for(int c = 0; c < cands; ++c)
            if(s.tries[c] > 0 && s.ns_per_pos[c] < s.ns_per_pos[best])
                best = c;
        if(++s.calls % 64 == 0)
        {
            // A neighbour of the best in one coordinate, in turn.
            const int turn = static_cast<int>(s.calls / 64) % 4;
            const int l = best % lens, g = best / lens;
            if(turn == 0 && l + 1 < lens) return g * lens + l + 1;
            if(turn == 1 && l > 0) return g * lens + l - 1;
            if(turn == 2 && g + 1 < grids) return (g + 1) * lens + l;
            if(turn == 3 && g > 0) return (g - 1) * lens + l;
        }
        return best;
    }

    void record(const int kind, const uint64_t pos, const int c, const double ms)
    {
        if(pos == 0 || c < 0)
            return;
        Slot& s = slot(kind, pos);
        const double v = 1e6 * ms / static_cast<double>(pos);
        s.ns_per_pos[c] = s.tries[c] == 0 ? v : 0.7 * s.ns_per_pos[c] + 0.3 * v;
        s.tries[c]++;
    }

private:
    struct Slot
    {
        double ns_per_pos[cands] = {};
        uint32_t tries[cands] = {};
        uint32_t calls = 0;
    };
    Slot slots_[3][64];

    Slot& slot(const int kind, const uint64_t pos)
    {
        int c = 0;
        while(c < 63 && (uint64_t(2) << c) <= pos)
            c++;
        return slots_[kind][c];
    }
};

}
