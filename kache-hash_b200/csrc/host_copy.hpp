// Host stores into page-locked staging buffers that the GPU then reads by DMA.
//
// A DMA read of host memory that host threads have just written runs slowly while the written lines sit dirty in
// those threads' private caches: on the B200 hosts measured, an 8 MB copy to the device of a page-locked buffer that
// 16 threads had just filled took 1.5-1.8 ms (about 5 GB/s), against 0.16-0.3 ms for the same buffer copied again
// unwritten, and 4.8 ms for 256 MB (55 GB/s). Streaming (non-temporal) stores write around the caches, so the lines
// are in memory when the copy engine reads them. Plain stores where the target has no streaming stores.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>

#if defined(__x86_64__) || defined(_M_X64)
#include <immintrin.h>
#define KACHE_B200_STREAM_STORES 1
#endif

namespace kache_b200
{

// Stores v at p (8-byte aligned) around the caches.
inline void stream_u64(uint64_t* p, const uint64_t v)
{
#ifdef KACHE_B200_STREAM_STORES
    _mm_stream_si64(reinterpret_cast<long long*>(p), static_cast<long long>(v));
#else
    *p = v;
#endif
}

// Makes this thread's streaming stores globally visible before its later stores (a worker calls it before it reports
// its part done, so that a copy issued after the whole pool returns reads them).
inline void stream_fence()
{
#ifdef KACHE_B200_STREAM_STORES
    _mm_sfence();
#endif
}

// Writes runs of bytes end to end from `dst` on: runs are collected in a small buffer and leave it in 16-byte
// streaming stores once the destination is 16-byte aligned; the bytes before that boundary and the last partial 16
// are written with plain stores. finish() writes what is left and fences.
class Stream_Writer
{
public:
    explicit Stream_Writer(char* dst) : dst_(dst), head_((16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15) {}
    Stream_Writer(const Stream_Writer&) = delete;
    Stream_Writer& operator=(const Stream_Writer&) = delete;

    void put(const char* src, size_t n)
    {
        while(n)
        {
            const size_t m = n < cap - fill_ ? n : cap - fill_;
            std::memcpy(buf_ + fill_, src, m);
            fill_ += m, src += m, n -= m;
            if(fill_ == cap)
                flush(false);
        }
    }

    void finish()
    {
        flush(true);
        stream_fence();
    }

    // Bytes written so far (flushed or not).
    size_t written() const { return total_ + fill_; }

private:
    static constexpr size_t cap = 4096;

    void flush(const bool last)
    {
        size_t at = 0;
        if(head_)
        {
            at = head_ < fill_ ? head_ : fill_;
            std::memcpy(dst_, buf_, at);
            dst_ += at, head_ -= at;
        }
        size_t body = (fill_ - at) / 16 * 16;
#ifdef KACHE_B200_STREAM_STORES
        for(size_t o = 0; o < body; o += 16)
            _mm_stream_si128(reinterpret_cast<__m128i*>(dst_ + o), _mm_loadu_si128(reinterpret_cast<const __m128i*>(buf_ + at + o)));
#else
        std::memcpy(dst_, buf_ + at, body);
#endif
        dst_ += body, at += body;
        const size_t rest = fill_ - at;
        total_ += at;
        if(last)
        {
            std::memcpy(dst_, buf_ + at, rest);
            dst_ += rest, total_ += rest, fill_ = 0;
        }
        else
        {
            std::memmove(buf_, buf_ + at, rest);
            fill_ = rest;
        }
    }

    alignas(16) char buf_[cap];
    size_t fill_ = 0;
    size_t total_ = 0;
    char* dst_;
    size_t head_;
};

}
