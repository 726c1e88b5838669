// The counter library on the GPU (counter/Kmer_Set_Counter.{hpp,cpp} in the reference): a fixed set of 31-mers,
// primed at count 0, whose 32-bit counts grow by one at each occurrence in the reads counted.
//
//   prime(path):     upsert with f(v) = v and 0 for absent k-mers            (Kmer_Set_Counter.cpp:63-74)
//   count(path):     present-only update with f(v) = v + 1, wrapping at 2^32  (Kmer_Set_Counter.cpp:77-93)
//   histogram(max):  the number of k-mers with each count in [1, max]         (Kmer_Set_Counter.cpp:96-119)
//   count_of(kmer):  a k-mer's count, 0 if absent or not ACGT                 (Kmer_Set_Counter.cpp:122-126)
// The table is <31, u32, 22> with its bucket count rounded up to a power of 2 (Kmer_Set_Counter.cpp:29-35).
// Files are read in batches of about 64 Mbp, the next batch parsed on a reader thread while the GPU works on the
// current one.
#include "engine.cuh"
#include "fastx.hpp"
#include "kache_b200.h"

#include <condition_variable>
#include <exception>
#include <mutex>
#include <new>
#include <thread>

namespace kache_b200
{
kache_table* make_table(uint32_t k, uint32_t l, uint32_t vb, uint64_t n, double lf, bool pow2);
}

struct kache_counter
{
    kache_table* t = nullptr;
    uint32_t threads = 1;
    ~kache_counter() { delete t; }
};

namespace
{

using namespace kache_b200;

constexpr size_t batch_bases = size_t(64) << 20;

template <typename F>
int guard(const F& f) noexcept
{
    try
    {
        return f();
    }
    catch(const std::bad_alloc&)
    {
        return KACHE_ENOMEM;
    }
    catch(const Cuda_Error&)
    {
        return KACHE_EINTERNAL;
    }
    catch(const std::runtime_error&)
    {
        return KACHE_EINVAL;    // Unreadable or malformed input; the reference throws std::runtime_error.
    }
    catch(...)
    {
        return KACHE_EINTERNAL;
    }
}

// Streams the file's batches to `f(seqs, lens, n)`, parsing the next batch while `f` runs on the current one.
template <typename F>
void for_batches(const char* path, const F& f)
{
    Fastx_Reader r(path);
    struct Slot { std::vector<char> bases; std::vector<size_t> lens; bool more = false; };
    Slot slot[2];
    slot[0].more = r.next(slot[0].bases, slot[0].lens, batch_bases);
    std::vector<const char*> seqs;
    for(int cur = 0; slot[cur].more; cur ^= 1)
    {
        std::exception_ptr err;
        Slot& nx = slot[cur ^ 1];
        std::thread reader([&](){ try { nx.more = r.next(nx.bases, nx.lens, batch_bases); } catch(...) { err = std::current_exception(); nx.more = false; } });
        Slot& s = slot[cur];
        seqs.resize(s.lens.size());
        size_t o = 0;
        for(size_t i = 0; i < s.lens.size(); ++i)
            seqs[i] = s.bases.data() + o, o += s.lens[i];
        try
        {
            f(seqs.data(), s.lens.data(), s.lens.size());
        }
        catch(...)
        {
            reader.join();
            throw;
        }
        reader.join();
        if(err)
            std::rethrow_exception(err);
    }
}

}

extern "C"
{

int kache_counter_new(const uint32_t k, const uint64_t n, const uint32_t threads, const double load_factor, kache_counter** const out) noexcept
{
    if(out == nullptr)
        return KACHE_EINVAL;
    *out = nullptr;
    // Kmer_Set_Counter.cpp:48-53: only 31-mers, and 1 to 128 threads.
    if(k != 31 || threads < 1 || threads > KACHE_MAX_USERS || !(load_factor > 0 && load_factor < 1) || !kache_b200::fits(n, load_factor, true))
        return KACHE_EINVAL;
    return guard([&]()
    {
        auto* c = new kache_counter;
        try
        {
            c->t = make_table(31, 22, 4, n, load_factor, true);
        }
        catch(...)
        {
            delete c;
            throw;
        }
        c->threads = threads;
        c->t->user_c = 1;
        *out = c;
        return KACHE_OK;
    });
}

void kache_counter_free(kache_counter* const c) noexcept
{
    delete c;
}

int kache_counter_prime(kache_counter* const c, const char* const path) noexcept
{
    if(c == nullptr || path == nullptr)
        return KACHE_EINVAL;
    return guard([&]()
    {
        for_batches(path, [&](const char* const* seqs, const size_t* lens, const size_t n){ c->t->upsert(0, seqs, lens, n, OP_KEEP, 0, 0); });
        return KACHE_OK;
    });
}

int kache_counter_count(kache_counter* const c, const char* const path, uint64_t* const found) noexcept
{
    if(c == nullptr || path == nullptr)
        return KACHE_EINVAL;
    return guard([&]()
    {
        uint64_t f = 0;
        for_batches(path, [&](const char* const* seqs, const size_t* lens, const size_t n){ f += c->t->update(seqs, lens, n, OP_ADD_WRAP, 1); });
        if(found)
            *found = f;
        return KACHE_OK;
    });
}

int kache_counter_prime_batch(kache_counter* const c, const char* const* const seqs, const size_t* const lens, const size_t n) noexcept
{
    if(c == nullptr || (n > 0 && (seqs == nullptr || lens == nullptr)))
        return KACHE_EINVAL;
    return guard([&](){ return c->t->upsert(0, seqs, lens, n, OP_KEEP, 0, 0), KACHE_OK; });
}

int kache_counter_count_batch(kache_counter* const c, const char* const* const seqs, const size_t* const lens, const size_t n, uint64_t* const found) noexcept
{
    if(c == nullptr || (n > 0 && (seqs == nullptr || lens == nullptr)))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const uint64_t f = c->t->update(seqs, lens, n, OP_ADD_WRAP, 1);
        if(found)
            *found = f;
        return KACHE_OK;
    });
}

int kache_counter_histogram(kache_counter* const c, const uint64_t max, uint64_t* const h) noexcept
{
    if(c == nullptr || h == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return c->t->histogram(max, h), KACHE_OK; });
}

int kache_counter_count_of(kache_counter* const c, const char* const kmer, uint64_t* const count) noexcept
{
    if(c == nullptr || kmer == nullptr || count == nullptr)
        return KACHE_EINVAL;
    return guard([&]()
    {
        uint64_t v = 0;
        *count = c->t->get(kmer, v) ? v : 0;
        return KACHE_OK;
    });
}

int kache_counter_size(kache_counter* const c, uint64_t* const n) noexcept
{
    if(c == nullptr || n == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return *n = c->t->size(), KACHE_OK; });
}

int kache_b200_fastx_read(const char* const path, const uint64_t batch, const kache_seqs_fn f, void* const ctx) noexcept
{
    if(path == nullptr || f == nullptr || batch == 0)
        return KACHE_EINVAL;
    return guard([&]()
    {
        Fastx_Reader r(path);
        std::vector<char> bases;
        std::vector<size_t> lens;
        std::vector<const char*> seqs;
        while(r.next(bases, lens, batch))
        {
            seqs.resize(lens.size());
            for(size_t i = 0, o = 0; i < lens.size(); o += lens[i], ++i)
                seqs[i] = bases.data() + o;
            if(f(ctx, seqs.data(), lens.data(), lens.size()) != 0)
                break;
        }
        return KACHE_OK;
    });
}

kache_table* kache_counter_table(kache_counter* const c) noexcept
{
    return c ? c->t : nullptr;
}

}
