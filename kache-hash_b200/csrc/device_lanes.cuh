// The streaming kernel, one lane per segment: each lane rolls its own stretch of a sequence base by base, as the
// reference's describers do per stretch (include/Kmer_Batch.hpp:191-250; its SIMD lanes, include/Kmer_Lanes.hpp:
// 164-244, take 4 stretches at once; a warp here takes 32), and hands each k-mer to the visitor.
//
// Per base, a lane updates the forward and reverse-complement k-mer and l-mer in registers (shifts and ORs), hashes
// the new canonical l-mer, and keeps the sliding minimum of the last w = k - l + 1 l-mer hashes with van Herk /
// Gil-Werman blocks of w: the prefix minimum of the current block in a register, the suffix minima of the previous
// block in shared memory (computed in place when a block completes). That is a constant three minimum operations
// per position whatever w is, and no branch that depends on the data, so the warp stays converged.
//
// Lanes of a warp work on 32 different segments -- for short reads, 32 different reads -- so their inserts rarely
// meet in one bucket. A warp steps as long as its longest segment; the host lists segments so that neighbours have
// similar lengths. Warps take their next 32 segments from a work counter (`next`, zeroed before the launch), so warps
// that drew short segments or fast probes take more, and the launch ends evenly however uneven the reads are.
#pragma once

#include "device_stream.cuh"

namespace kache_b200
{

constexpr int lane_block = 256;     // Threads per block of the lane kernel.

template <int k, int l, typename Visitor>
__global__ void __launch_bounds__(lane_block, 4) lane_kernel(const Dev_Batch batch, const uint64_t seg_b, const uint64_t seg_e, unsigned long long* next, Visitor vis)
{
    constexpr int w = k - l + 1;
    static_assert(k <= 32 && l <= k && w >= 1, "k-mers in a machine word");
    constexpr uint64_t kmask = (k == 32 ? ~0ull : (1ull << (2 * k)) - 1);
    constexpr uint64_t lmask = (l == 32 ? ~0ull : (1ull << (2 * l)) - 1);
    __shared__ uint64_t blk[w][lane_block];     // This thread's column: the current block's l-mer hashes, then suffix minima.
    __shared__ uint4 csc[2][lane_block];        // This thread's copy of its last primary bucket's checksums.
    const uint32_t lane = threadIdx.x & 31;
    vis.begin();
    vis.lane_cache(&csc[0][threadIdx.x], &csc[1][threadIdx.x]);

    const auto take = [&]() -> uint64_t
    {
        unsigned long long g = 0;
        if(lane == 0)
            g = atomicAdd(next, 32ull);
        return seg_b + __shfl_sync(0xFFFFFFFFu, g, 0);
    };
    for(uint64_t g0 = take(); g0 < seg_e; g0 = take())
    {
        const uint64_t g = g0 + lane;
        const bool has = g < seg_e;
        uint64_t q = 0, p0 = 0, obase = 0;
        uint32_t npos = 0, steps = 0;
        const uint8_t* p = nullptr;
        if(has)
        {
            const uint64_t packed = batch.segs[g];
            q = packed >> 24;
            const uint64_t b0 = batch.off[q], len = batch.off[q + 1] - b0;
            p0 = (packed & 0xFFFFFF) * batch.seg_len;
            obase = batch.pos_off[q] + p0;
            npos = static_cast<uint32_t>(min(len - k + 1 - p0, static_cast<uint64_t>(batch.seg_len)));
            p = batch.seq(q, b0) + p0;
            steps = npos + k - 1;
        }
        const uint32_t wsteps = __reduce_max_sync(0xFFFFFFFFu, steps);
        vis.lane_begin(q, has);

        uint64_t kf = 0, kr = 0, lf = 0, lr = 0, pm = ~0ull;
        uint32_t run = 0, bj = 0;
        for(uint32_t t = 0; t < wsteps; ++t)
        {
            const uint32_t ch = t < steps ? p[t] : 0u;
            const uint32_t x = (ch | 0x20u) - 'a';
            const bool ok = x < 20u && ((0x80045u >> x) & 1u);  // a, c, g, t
            run = ok ? run + 1 : 0;
            const uint64_t b = ((ch >> 2) ^ (ch >> 1)) & 3u;
            kf = ((kf << 2) | b) & kmask;
            kr = (kr >> 2) | ((3 - b) << (2 * (k - 1)));
            lf = ((lf << 2) | b) & lmask;
            lr = (lr >> 2) | ((3 - b) << (2 * (l - 1)));
            if(t + 1 < l)
                continue;

            // The l-mer ending here; the window of the last w of them.
            const uint64_t hc = wang_u64(min64(lf, lr));
            pm = min64(pm, hc);
            uint64_t h = pm;
            if(bj + 1 < w)
                h = min64(h, blk[bj + 1][threadIdx.x]);
            blk[bj][threadIdx.x] = hc;
            if(++bj == w)
            {
                bj = 0, pm = ~0ull;
                uint64_t m = blk[w - 1][threadIdx.x];
#pragma unroll
                for(int j = w - 2; j >= 0; --j)
                    m = min64(m, blk[j][threadIdx.x]), blk[j][threadIdx.x] = m;
            }
            if(t + 1 < k)
                continue;

            Kmer_Desc d;
            const uint32_t i = t + 1 - k;
            d.q = q;
            d.pos = p0 + i;
            d.out = obase + i;
            d.last = false;
            d.in = i < npos;
            d.valid = d.in && run >= static_cast<uint32_t>(k);
            d.key = min64(kf, kr);
            d.fwd = kf <= kr;
            d.c = checksum_of(d.key);
            d.h = h;
            vis.visit(d, lane);
        }
        vis.lane_end(q, has);
    }
    vis.end(lane);
}

}
