// Per-sequence counts over a batch already in device memory, for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc on the path where they query the table: code running inside a memory pool
// whose allocator must not be re-entered, or an embedding process that budgets every byte of HBM itself.
// kache_b200_count_dev allocates the scratch it needs (segment lists, scan buffers) on first use and whenever a batch
// outgrows it. This variant does the same counting
// with its scratch in one fixed array below, which every GPU that loads the library holds until the process exits,
// and calls no cudaMalloc, cudaFree or allocating library routine.
//
// The scratch array is shared by every call: each call clears the part that must start at zero. Two calls whose
// work overlaps on the GPU (from different streams or threads) race on it; serialise them.
#include "engine.cuh"
#include "kache_b200.h"

#include <mutex>

namespace
{

using namespace kache_b200;

// 8 MiB: a header, then up to 1,048,544 segments of up to 512 k-mer positions each.
constexpr size_t noalloc_scratch_bytes = size_t(8) << 20;
constexpr size_t noalloc_header_bytes = 256;
constexpr uint64_t noalloc_max_segments = (noalloc_scratch_bytes - noalloc_header_bytes) / sizeof(uint64_t);
static_assert(noalloc_max_segments == KACHE_B200_NOALLOC_MAX_SEGMENTS, "the header states the same maximum");

static __device__ __align__(256) unsigned char noalloc_scratch[noalloc_scratch_bytes];

// The scratch as the kernels use it: [0, 8) the number of segments claimed, [8, 12) set if a batch had more
// segments than fit, [256, ...) the segments (q << 24 | s).
struct Scratch
{
    unsigned long long* count;
    unsigned int* overflow;
    uint64_t* segs;
};

Scratch scratch_at(void* base)
{
    char* p = static_cast<char*>(base);
    return Scratch{reinterpret_cast<unsigned long long*>(p), reinterpret_cast<unsigned int*>(p + 8), reinterpret_cast<uint64_t*>(p + noalloc_header_bytes)};
}

// Lists each sequence's segments, claiming a range of the list per sequence; the order does not matter to counts.
__global__ void noalloc_segments_kernel(const uint64_t* off, const uint64_t n, const int k, const Scratch s)
{
    const uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(q >= n)
        return;
    const uint64_t len = off[q + 1] - off[q];
    const uint64_t p = len >= uint64_t(k) ? len - k + 1 : 0;
    const uint64_t nseg = (p + seg_positions - 1) / seg_positions;
    if(nseg == 0)
        return;
    if(nseg - 1 > max_seg_index)
    {
        atomicOr(s.overflow, 1u);   // Segment indexes take 24 bits of an entry: a longer sequence cannot be listed.
        return;
    }
    const uint64_t at = atomicAdd(s.count, static_cast<unsigned long long>(nseg));
    if(at + nseg > noalloc_max_segments)
    {
        atomicOr(s.overflow, 1u);
        return;
    }
    for(uint64_t i = 0; i < nseg; ++i)
        s.segs[at + i] = (q << 24) | i;
}

// The streaming kernel's segment loop (device_stream.cuh) over the listed segments, with the per-sequence count
// visitor; the segment count comes from the scratch. A batch that did not fit (the overflow flag) is not counted at
// all: a sequence whose claim ran past the end wrote none of the entries it claimed, so entries below the end may
// still hold an earlier call's segments, whose sequence indexes need not exist in this batch.
template <int k, int l, bool set_>
__global__ void __launch_bounds__(32 * stream_warps) noalloc_count_kernel(const Dev_Table T, const uint8_t* bases, const uint64_t* off, const Scratch s, unsigned long long* counts)
{
    constexpr int w = k - l + 1;
    __shared__ uint64_t ring_all[stream_warps][64];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t* ring = ring_all[wid];
    if(*s.overflow)
        return;
    Seq_Reduce_Visitor<set_, uint8_t, 0> vis{T, counts, 0, 0, 0, 0};
    vis.begin();

    const uint64_t nsegs = min(static_cast<uint64_t>(*s.count), noalloc_max_segments);
    const uint64_t warps = uint64_t(gridDim.x) * stream_warps;
    for(uint64_t g = uint64_t(blockIdx.x) * stream_warps + wid; g < nsegs; g += warps)
    {
        const uint64_t packed = s.segs[g];
        const uint64_t q = packed >> 24, sg = packed & 0xFFFFFF;
        const uint64_t b0 = off[q], len = off[q + 1] - b0;
        const uint8_t* seq = bases + b0;
        const uint64_t npos = len - k + 1;
        const uint64_t p0 = sg * seg_positions;
        const uint64_t p1 = min(npos, p0 + seg_positions);
        const uint32_t rows = static_cast<uint32_t>((p1 - p0 + 31) / 32);
        const uint8_t* sp = seq + p0 + lane;
        const int32_t rem = static_cast<int32_t>(min(len - p0, uint64_t(1) << 30)) - static_cast<int32_t>(lane);

        Row r0 = load_row(sp, rem, 0, lane);
        Row r1 = load_row(sp, rem, 32, lane);
        {
            uint64_t f, rc;
            window<l>(r0, r1, lane, f, rc);
            ring[lane] = wang_u64(f < rc ? f : rc);
        }
        vis.begin_segment(q);
        for(uint32_t r = 0; r < rows; ++r)
        {
            const Row r2 = load_row(sp, rem, 32 * (r + 2), lane);
            {
                uint64_t f, rc;
                window<l>(r1, r2, lane, f, rc);
                ring[((r + 1) & 1) * 32 + lane] = wang_u64(f < rc ? f : rc);
            }
            __syncwarp();
            Kmer_Desc d;
            uint64_t f, rc;
            window<k>(r0, r1, lane, f, rc);
            const uint64_t vbits = ((uint64_t(r1.valid) << 32) | r0.valid) >> lane;
            const uint64_t km = (k == 32 ? 0xFFFFFFFFull : (1ull << k) - 1);
            d.pos = p0 + 32 * r + lane;
            d.q = q;
            d.in = d.pos < p1;
            d.valid = d.in && (vbits & km) == km;
            d.key = f < rc ? f : rc;
            d.fwd = f <= rc;
            d.c = checksum_of(d.key);
            uint64_t h = ~0ull;
            const uint32_t base = (r & 1) * 32 + lane;
#pragma unroll
            for(int x = 0; x < w; ++x)
            {
                const uint64_t v = ring[(base + x) & 63];
                h = v < h ? v : h;
            }
            d.h = h;
            vis.visit(d, lane);
            __syncwarp();
            r0 = r1, r1 = r2;
        }
        vis.end_segment(q, lane);
    }
}

// The scratch's device address, looked up once per device with that device current. In host code the array's
// name stands for a host-side shadow, not for device memory, so kernels get this address instead.
std::mutex scratch_mu;
void* scratch_addr[256] = {};

cudaError_t scratch_on(const int dev, void** out)
{
    if(dev < 0 || dev >= 256)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(scratch_mu);
    if(scratch_addr[dev] == nullptr)
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
        if(e != cudaSuccess)
            return e;
        scratch_addr[dev] = p;
    }
    *out = scratch_addr[dev];
    return cudaSuccess;
}

}

extern "C" int kache_b200_count_dev_noalloc(kache_table* const t, const uint8_t* const d_bases, const uint64_t* const d_off, const uint64_t n, uint64_t* const d_counts) noexcept
{
    if(t == nullptr || (n > 0 && (d_bases == nullptr || d_off == nullptr || d_counts == nullptr)) || t->kmer_k != 31 || t->kmer_l != 22)
        return KACHE_EINVAL;
    if(n > noalloc_max_segments)
        return KACHE_EINVAL;    // More sequences than the scratch can list segments for.
    if(n == 0)
        return KACHE_OK;
    try
    {
        std::lock_guard<std::mutex> g(t->work);
        int dev = 0;
        if(cudaGetDevice(&dev) != cudaSuccess)
            return KACHE_EINTERNAL;
        void* base = nullptr;
        if(scratch_on(dev, &base) != cudaSuccess)
            return KACHE_EINTERNAL;
        const Scratch s = scratch_at(base);
        const cudaStream_t st = t->stream();
        const Dev_Table T = t->device_table();
        // The header starts at zero; the counts are the caller's output, zeroed here.
        if(cudaMemsetAsync(base, 0, noalloc_header_bytes, st) != cudaSuccess || cudaMemsetAsync(d_counts, 0, n * sizeof(uint64_t), st) != cudaSuccess)
            return KACHE_EINTERNAL;
        noalloc_segments_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(d_off, n, 31, s);
        launches()++;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const unsigned blocks = static_cast<unsigned>(uint64_t(sms) * 16);
        if(t->value_bytes == 0)
            noalloc_count_kernel<31, 22, true><<<blocks, 32 * stream_warps, 0, st>>>(T, d_bases, d_off, s, reinterpret_cast<unsigned long long*>(d_counts));
        else
            noalloc_count_kernel<31, 22, false><<<blocks, 32 * stream_warps, 0, st>>>(T, d_bases, d_off, s, reinterpret_cast<unsigned long long*>(d_counts));
        launches()++;
        if(cudaGetLastError() != cudaSuccess)
            return KACHE_EINTERNAL;
        unsigned int overflow = 0;
        if(cudaMemcpyAsync(&overflow, s.overflow, sizeof(overflow), cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
            return KACHE_EINTERNAL;
        return overflow ? KACHE_EINVAL : KACHE_OK;
    }
    catch(...)
    {
        return KACHE_EINTERNAL;
    }
}
