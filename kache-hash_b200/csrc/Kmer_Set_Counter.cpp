// The reference's C++ counter class (counter/Kmer_Set_Counter.hpp:23-76) over the B200 counter's C functions
// (kache_counter_*, csrc/counter.cu): argument checks and exceptions as the reference's constructor makes them
// (counter/Kmer_Set_Counter.cpp:48-53), phase timings as it keeps them.
#include "Kmer_Set_Counter.hpp"
#include "kache_b200.h"

#include <chrono>
#include <new>
#include <stdexcept>

namespace kache_hash
{

namespace
{

constexpr uint16_t counter_k = 31;
constexpr std::size_t max_thread_c = 128;   // As many users as a table takes.

double seconds_since(const std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Turns a failed call's status into the exception a C++ caller of the reference would catch.
void check(const int code, const std::string& what)
{
    if(code == KACHE_OK)
        return;
    if(code == KACHE_ENOMEM)
        throw std::bad_alloc();
    throw std::runtime_error(what + ": " + kache_strerror(code));
}

}

struct Kmer_Set_Counter::Impl
{
    kache_counter* c = nullptr;
    Timings timings;

    ~Impl() { kache_counter_free(c); }
};

bool Kmer_Set_Counter::supports(const uint16_t k)
{
    return k == counter_k;
}

Kmer_Set_Counter::Kmer_Set_Counter(const uint16_t k, const std::size_t n, const std::size_t thread_c, const double lf)
{
    if(!supports(k))
        throw std::invalid_argument("k-mers of length " + std::to_string(k) + " are not supported, only of " + std::to_string(counter_k));
    if(thread_c < 1 || thread_c > max_thread_c)
        throw std::invalid_argument("the thread count must be in [1, " + std::to_string(max_thread_c) + "]");
    if(!(lf > 0 && lf < 1))
        throw std::invalid_argument("the load factor must be in (0, 1)");

    const auto t0 = std::chrono::steady_clock::now();
    impl = std::make_unique<Impl>();
    const int r = kache_counter_new(k, n, static_cast<uint32_t>(thread_c), lf, &impl->c);
    if(r == KACHE_EINVAL)
        throw std::invalid_argument("a table for " + std::to_string(n) + " k-mers at load factor " + std::to_string(lf) + " is too large");
    check(r, "creating the counter");
    impl->timings.alloc = seconds_since(t0);
}

Kmer_Set_Counter::~Kmer_Set_Counter() = default;

void Kmer_Set_Counter::prime(const std::string& path)
{
    const auto t0 = std::chrono::steady_clock::now();
    check(kache_counter_prime(impl->c, path.c_str()), "priming from " + path);
    impl->timings.prime += seconds_since(t0);
}

std::size_t Kmer_Set_Counter::count(const std::string& path)
{
    const auto t0 = std::chrono::steady_clock::now();
    uint64_t found = 0;
    check(kache_counter_count(impl->c, path.c_str(), &found), "counting from " + path);
    impl->timings.count += seconds_since(t0);
    return static_cast<std::size_t>(found);
}

std::vector<std::size_t> Kmer_Set_Counter::histogram(const std::size_t max)
{
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<uint64_t> h(max + 1, 0);
    check(kache_counter_histogram(impl->c, max, h.data()), "histogram");
    impl->timings.histogram += seconds_since(t0);
    return std::vector<std::size_t>(h.begin(), h.end());
}

uint64_t Kmer_Set_Counter::count_of(const char* const kmer) const
{
    uint64_t c = 0;
    check(kache_counter_count_of(impl->c, kmer, &c), "count_of");
    return c;
}

std::size_t Kmer_Set_Counter::size() const
{
    uint64_t n = 0;
    check(kache_counter_size(impl->c, &n), "size");
    return static_cast<std::size_t>(n);
}

const Kmer_Set_Counter::Timings& Kmer_Set_Counter::timings() const
{
    return impl->timings;
}

}
