// The counter library's C++ surface, with the reference's class, namespace and signatures
// (counter/Kmer_Set_Counter.hpp:23-76), over the B200 counter of kache_b200.h (kache_counter_*): a C++ caller of
// the reference's Kmer_Set_Counter (PanGenie-style k-mer set counting) recompiles against this header and links
// libkache_b200 instead. The table lives in HBM; files are read on the host and their batches counted on the GPU.
#ifndef KACHE_HASH_KMER_SET_COUNTER_HPP
#define KACHE_HASH_KMER_SET_COUNTER_HPP

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace kache_hash
{

// Counter of the canonical 31-mers of reads that belong to a set fixed beforehand (counter/Kmer_Set_Counter.hpp:
// 17-22). Inputs are FASTA or FASTQ files (or pipes); non-ACGT characters split their sequences. Counts are 32-bit
// and wrap. The counter's operations must not overlap one another, but for histograms and count_ofs.
class Kmer_Set_Counter
{
private:

    struct Impl;
    std::unique_ptr<Impl> impl;

public:

    // Time taken by the phases, in seconds (counter/Kmer_Set_Counter.hpp:31-38): `alloc` is the table's creation in
    // HBM; the others include reading the files.
    struct Timings
    {
        double alloc = 0;
        double prime = 0;
        double count = 0;
        double histogram = 0;
    };

    // Whether k-mers of length `k` are supported: only 31-mers are (counter/Kmer_Set_Counter.cpp:42-45).
    static bool supports(uint16_t k);

    // A counter of `k`-mers with room for `n` k-mers at load factor `lf`, beyond which it grows, its bucket count
    // rounded up to a power of 2, and `thread_c` in [1, 128] threads (counter/Kmer_Set_Counter.cpp:48-57). Throws
    // std::invalid_argument for another k, a thread count outside [1, 128] or a load factor outside (0, 1), and
    // std::bad_alloc when the device has no room for the table.
    Kmer_Set_Counter(uint16_t k, std::size_t n, std::size_t thread_c, double lf = 0.9);

    ~Kmer_Set_Counter();

    Kmer_Set_Counter(const Kmer_Set_Counter&) = delete;
    Kmer_Set_Counter& operator=(const Kmer_Set_Counter&) = delete;

    // Adds the k-mers of the sequences of the FASTA or FASTQ file at `path` to the set with count 0; present ones keep
    // their counts (counter/Kmer_Set_Counter.cpp:63-74). Throws std::runtime_error if the file cannot be read or
    // parsed.
    void prime(const std::string& path);

    // Increments the count of each k-mer of the reads at `path` that is in the set, at each of its occurrences, and
    // returns the occurrences counted (counter/Kmer_Set_Counter.cpp:77-93). Throws as `prime`.
    std::size_t count(const std::string& path);

    // The histogram of the counts: at index c the number of k-mers with count c, for c in [1, max], 0 at index 0
    // (counter/Kmer_Set_Counter.cpp:96-119).
    std::vector<std::size_t> histogram(std::size_t max);

    // The count of the k-mer of the 31 characters at `kmer`: 0 if it is not in the set, as for one with a non-ACGT
    // character (counter/Kmer_Set_Counter.cpp:122-126).
    uint64_t count_of(const char* kmer) const;

    // The number of k-mers in the set.
    std::size_t size() const;

    // The time taken by the phases so far.
    const Timings& timings() const;
};

}

#endif
