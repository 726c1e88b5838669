// The device's memory roofs for the table's access patterns, the GPU analog of the reference's roof tool
// (tools/memory-roof.cpp:21-29): sequential reads, independent random reads and updates of 32-byte sectors, and
// dependent random reads (a chase whose rate per thread is the inverse of the memory latency), over an array as large
// as the tables the roofs bound. The table kernels touch HBM a sector at a time at random, so their achievable
// bandwidth is the random-sector roof rather than a streaming copy's.
#include "engine.cuh"
#include "kache_b200.h"

namespace kache_b200
{
namespace
{

__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    return mix64(x);
}

constexpr int roof_block = 256;
constexpr int roof_unroll = 8;     // Independent accesses a thread keeps in flight.

__global__ void __launch_bounds__(roof_block) roof_seq_read(const uint4* a, const uint64_t n16, unsigned long long* sink)
{
    uint32_t acc = 0;
    const uint64_t stride = uint64_t(gridDim.x) * roof_block;
    for(uint64_t i = uint64_t(blockIdx.x) * roof_block + threadIdx.x; i < n16; i += stride)
    {
        const uint4 v = __ldcs(a + i);
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if(acc == 0x9E3779B9u)
        atomicAdd(sink, 1ull);
}

// Each thread: `per` sector reads (kind 1) or atomic adds (kind 2) at random sectors, roof_unroll at a time.
template <int kind_>
__global__ void __launch_bounds__(roof_block) roof_random(uint4* a, const uint64_t mask, const uint32_t per, const uint64_t seed, unsigned long long* sink)
{
    const uint64_t t = uint64_t(blockIdx.x) * roof_block + threadIdx.x;
    uint32_t acc = 0;
    for(uint32_t i = 0; i < per; i += roof_unroll)
    {
        uint64_t s[roof_unroll];
#pragma unroll
        for(int u = 0; u < roof_unroll; ++u)
            s[u] = splitmix64(seed ^ (t * per + i + u)) & mask;
        if constexpr(kind_ == 1)
        {
            // One 16-byte load per sector: HBM moves the whole 32-byte sector either way.
            uint4 v[roof_unroll];
#pragma unroll
            for(int u = 0; u < roof_unroll; ++u)
                v[u] = __ldcg(a + 2 * s[u]);
#pragma unroll
            for(int u = 0; u < roof_unroll; ++u)
                acc ^= v[u].x ^ v[u].w;
        }
        else
        {
#pragma unroll
            for(int u = 0; u < roof_unroll; ++u)
                atomicAdd(reinterpret_cast<unsigned long long*>(a + 2 * s[u]), 1ull);
        }
    }
    if(acc == 0x9E3779B9u)
        atomicAdd(sink, 1ull);
}

// Sector s holds, in its first word, the index of a random next sector.
__global__ void roof_chase_init(uint4* a, const uint64_t sectors, const uint64_t mask)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for(uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < sectors; s += stride)
        *reinterpret_cast<unsigned long long*>(a + 2 * s) = splitmix64(s * 0xD6E8FEB86659FD93ull) & mask;
}

__global__ void __launch_bounds__(roof_block) roof_chase(const uint4* a, const uint64_t mask, const uint32_t per, unsigned long long* sink)
{
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    uint64_t s = splitmix64(t) & mask;
    for(uint32_t i = 0; i < per; ++i)
        s = __ldcg(reinterpret_cast<const unsigned long long*>(a + 2 * s)) & mask;
    if(s == 0x9E3779B9u)
        atomicAdd(sink, 1ull);
}

}
}

using namespace kache_b200;

extern "C" int kache_b200_memory_roof(const uint64_t bytes, const uint32_t kind, const uint64_t accesses, double* const ms, double* const rate) noexcept
{
    if(ms == nullptr || rate == nullptr || kind > 3 || bytes < (uint64_t(1) << 20) || (kind != 0 && accesses == 0))
        return KACHE_EINVAL;
    uint64_t sectors = 1;
    while(sectors * 2 * 32 <= bytes)
        sectors *= 2;
    const uint64_t mask = sectors - 1;
    uint4* a = nullptr;
    unsigned long long* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = KACHE_OK;
    try
    {
        int dev = 0, sms = 148;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
        check(cudaMalloc(&a, sectors * 32), "cudaMalloc");
        check(cudaMalloc(&sink, 8), "cudaMalloc");
        check(cudaMemset(a, 0, sectors * 32), "memset");
        check(cudaEventCreate(&e0), "event"), check(cudaEventCreate(&e1), "event");
        const unsigned blocks = static_cast<unsigned>(sms) * 8;    // 2048 threads per SM.
        const uint64_t threads = kind == 3 ? uint64_t(sms) * 32 : uint64_t(blocks) * roof_block;
        uint32_t per = static_cast<uint32_t>(std::max<uint64_t>(1, (accesses + threads - 1) / threads));
        if(kind == 1 || kind == 2)
            per = (per + roof_unroll - 1) / roof_unroll * roof_unroll;
        if(kind == 3)
        {
            roof_chase_init<<<blocks, roof_block>>>(a, sectors, mask);
            launches()++;
        }
        float t = 0;
        for(int rep = 0; rep < 2; ++rep)   // A warm-up, then the timed run.
        {
            check(cudaEventRecord(e0), "event");
            switch(kind)
            {
            case 0: roof_seq_read<<<blocks, roof_block>>>(a, sectors * 2, sink); break;
            case 1: roof_random<1><<<blocks, roof_block>>>(a, mask, per, 0x2545F4914F6CDD1Dull + rep, sink); break;
            case 2: roof_random<2><<<blocks, roof_block>>>(a, mask, per, 0x2545F4914F6CDD1Dull + rep, sink); break;
            default: roof_chase<<<static_cast<unsigned>(sms), 32>>>(a, mask, per, sink); break;  // A warp per SM: the unloaded latency.
            }
            launches()++;
            check(cudaGetLastError(), "launch");
            check(cudaEventRecord(e1), "event");
            check(cudaEventSynchronize(e1), "event sync");
            check(cudaEventElapsedTime(&t, e0, e1), "event time");
        }
        *ms = t;
        // Sequential: bytes per second. Random reads and updates: sectors per second. Chase: dependent loads per
        // second of one warp per SM (the latency is those threads / rate).
        const double done = kind == 0 ? static_cast<double>(sectors * 32) : static_cast<double>(threads) * per;
        *rate = done / (t * 1e-3);
    }
    catch(const std::bad_alloc&)
    {
        rc = KACHE_ENOMEM;
    }
    catch(...)
    {
        rc = KACHE_EINTERNAL;
    }
    if(e0)
        cudaEventDestroy(e0);
    if(e1)
        cudaEventDestroy(e1);
    if(a)
        cudaFree(a);
    if(sink)
        cudaFree(sink);
    return rc;
}
