// Checks of the counter's C++ surface (include/Kmer_Set_Counter.hpp) against an exact brute-force count, after the
// reference's counter test (test/counter.cpp:374-497): a set primed from a FASTA file of several-line records (a
// genome in mixed case with N's, and short variant stretches), counted from FASTQ reads drawn from it on either strand
// with errors, from a file and from a pipe; priming again keeps the counts; count_of of every set k-mer in both
// orientations, in lower case and with an N, and of absent k-mers; histograms of bounds 3 and 10000; sizes and the
// occurrences counted; the constructor's invalid arguments. Built by kache-hash_b200/build.py; run by
// tests/test_gpu_counter_cpp.py with a scratch directory. Prints one line per configuration, exits 0 iff all agree.
#include "Kmer_Set_Counter.hpp"

#include <sys/stat.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

using kache_hash::Kmer_Set_Counter;

constexpr int k = 31;

static uint64_t state = 0x2545F4914F6CDD1Dull;
static uint64_t next() { state ^= state << 13, state ^= state >> 7, state ^= state << 17; return state; }
static std::size_t below(const std::size_t n) { return next() % n; }

static std::string random_bases(const std::size_t len, const char* alpha, const std::size_t m)
{
    std::string s(len, 'A');
    for(auto& c : s)
        c = alpha[below(m)];
    return s;
}

static char complement(const char c)
{
    switch(c | 0x20)
    {
    case 'a': return 'T';
    case 'c': return 'G';
    case 'g': return 'C';
    case 't': return 'A';
    default: return 'N';
    }
}

static std::string revcomp(const std::string& s)
{
    std::string r(s.rbegin(), s.rend());
    for(auto& c : r)
        c = complement(c);
    return r;
}

// The canonical 2-bit encoding of the k characters at s, or -1 if one is not ACGT (either case).
static int64_t canonical(const char* s)
{
    uint64_t f = 0, r = 0;
    for(int i = 0; i < k; ++i)
    {
        uint64_t b;
        switch(s[i] | 0x20)
        {
        case 'a': b = 0; break;
        case 'c': b = 1; break;
        case 'g': b = 2; break;
        case 't': b = 3; break;
        default: return -1;
        }
        f = (f << 2) | b;
        r |= (3 - b) << (2 * i);
    }
    return static_cast<int64_t>(f < r ? f : r);
}

static std::string decode(uint64_t x)
{
    std::string s(k, 'A');
    for(int i = k - 1; i >= 0; --i, x >>= 2)
        s[i] = "ACGT"[x & 3];
    return s;
}

static void write_file(const std::string& path, const std::string& text)
{
    std::ofstream(path, std::ios::binary) << text;
}

int main(int argc, char** argv)
{
    if(argc < 2)
    {
        std::fprintf(stderr, "usage: counter_check <scratch-dir>\n");
        return 2;
    }
    const std::string dir = argv[1];

    // The set's sequences: chromosomes in mixed case with N's, and variants of short stretches of them.
    std::vector<std::string> set_seqs;
    for(int i = 0; i < 8; ++i)
    {
        auto g = random_bases(25'000, "ACGTACGTACGTacgt", 16);
        for(int j = 0; j < 15; ++j)
            g[below(g.size())] = 'N';
        set_seqs.push_back(g);
    }
    for(int i = 0; i < 1500; ++i)
    {
        const auto& g = set_seqs[below(8)];
        const std::size_t len = 35 + below(70);
        auto v = g.substr(below(g.size() - len), len);
        v[below(len)] = "ACGT"[below(4)];
        set_seqs.push_back(v);
    }
    // The reads: stretches of the set's sequences on either strand with a few errors or N's, and random reads.
    std::vector<std::string> reads;
    for(int i = 0; i < 25'000; ++i)
    {
        std::string s;
        if(below(5) == 0)
            s = random_bases(120, "ACGT", 4);
        else
        {
            const auto& g = set_seqs[below(set_seqs.size())];
            const std::size_t len = std::min<std::size_t>(120, g.size());
            s = g.substr(below(g.size() - len + 1), len);
            if(below(2))
                s = revcomp(s);
            for(std::size_t e = below(3); e > 0; --e)
                s[below(s.size())] = "ACGTN"[below(5)];
        }
        reads.push_back(s);
    }

    // FASTA with 70-column lines; FASTQ with one line per sequence.
    std::string fa, fq;
    for(std::size_t i = 0; i < set_seqs.size(); ++i)
    {
        fa += ">s" + std::to_string(i) + "\n";
        for(std::size_t o = 0; o < set_seqs[i].size(); o += 70)
            fa += set_seqs[i].substr(o, 70) + "\n";
    }
    for(std::size_t i = 0; i < reads.size(); ++i)
        fq += "@r" + std::to_string(i) + "\n" + reads[i] + "\n+\n" + std::string(reads[i].size(), 'I') + "\n";
    const std::string set_path = dir + "/set.fa", reads_path = dir + "/reads.fq", pipe_path = dir + "/reads.pipe";
    write_file(set_path, fa);
    write_file(reads_path, fq);

    // The exact count.
    std::unordered_map<uint64_t, uint64_t> C;
    for(const auto& s : set_seqs)
        for(std::size_t i = 0; i + k <= s.size(); ++i)
            if(const int64_t x = canonical(s.data() + i); x >= 0)
                C[static_cast<uint64_t>(x)] = 0;
    std::size_t found_exp = 0;
    for(const auto& s : reads)
        for(std::size_t i = 0; i + k <= s.size(); ++i)
            if(const int64_t x = canonical(s.data() + i); x >= 0)
                if(auto it = C.find(static_cast<uint64_t>(x)); it != C.end())
                    it->second++, found_exp++;
    const auto hist = [&](const std::size_t max)
    {
        std::vector<std::size_t> H(max + 1, 0);
        for(const auto& kv : C)
            if(kv.second >= 1 && kv.second <= max)
                H[kv.second]++;
        return H;
    };

    int fail = 0;
    struct Config { std::size_t n, threads; bool pipe; };
    for(const Config cfg : {Config{1000, 1, false}, Config{C.size(), 16, false}, Config{C.size(), 128, true}})
    {
        Kmer_Set_Counter K(k, cfg.n, cfg.threads);
        K.prime(set_path);
        const std::size_t primed = K.size();
        std::size_t found = 0;
        if(!cfg.pipe)
            found = K.count(reads_path);
        else
        {
            unlink(pipe_path.c_str());
            mkfifo(pipe_path.c_str(), 0600);
            std::thread w([&](){ write_file(pipe_path, fq); });
            found = K.count(pipe_path);
            w.join();
        }
        K.prime(set_path);      // Priming again leaves the counts.

        std::size_t wrong = 0;
        for(const auto& kv : C)
        {
            std::string s = decode(kv.first);
            wrong += K.count_of(s.c_str()) != kv.second;
            wrong += K.count_of(revcomp(s).c_str()) != kv.second;
            for(auto& c : s)
                c = static_cast<char>(c | 0x20);
            wrong += K.count_of(s.c_str()) != kv.second;
            s[kv.first % k] = 'N';
            wrong += K.count_of(s.c_str()) != 0;
        }
        for(int i = 0; i < 5000; ++i)
        {
            const std::string s = random_bases(k, "ACGT", 4);
            if(!C.count(static_cast<uint64_t>(canonical(s.c_str()))))
                wrong += K.count_of(s.c_str()) != 0;
        }
        const bool hist_ok = K.histogram(3) == hist(3) && K.histogram(10'000) == hist(10'000);
        const bool ok = primed == C.size() && K.size() == C.size() && found == found_exp && wrong == 0 && hist_ok;
        const auto& t = K.timings();
        std::printf("counter n %zu, %zu threads%s: size %zu (exact %zu), found %zu (exact %zu), %zu wrong lookups, histograms %s; "
                    "%.3f s alloc, %.3f s prime, %.3f s count, %.3f s histogram: %s\n",
                    cfg.n, cfg.threads, cfg.pipe ? ", reads from a pipe" : "", K.size(), C.size(), found, found_exp, wrong,
                    hist_ok ? "equal" : "DIFFER", t.alloc, t.prime, t.count, t.histogram, ok ? "ok" : "WRONG");
        fail += !ok;
    }

    int caught = 0;
    try { Kmer_Set_Counter K(27, 1000, 1); } catch(const std::invalid_argument&) { caught++; }
    try { Kmer_Set_Counter K(k, 1000, 0); } catch(const std::invalid_argument&) { caught++; }
    try { Kmer_Set_Counter K(k, 1000, 129); } catch(const std::invalid_argument&) { caught++; }
    bool unreadable = false;
    try { Kmer_Set_Counter K(k, 1000, 1); K.prime(dir + "/absent.fa"); } catch(const std::runtime_error&) { unreadable = true; }
    const bool sup = Kmer_Set_Counter::supports(31) && !Kmer_Set_Counter::supports(27);
    std::printf("counter arguments: %d of 3 invalid ones rejected, unreadable file %s, supports(31) and not (27): %s\n", caught,
                unreadable ? "rejected" : "NOT REJECTED", sup ? "yes" : "NO");
    fail += caught != 3 || !unreadable || !sup;
    std::printf("%s\n", fail ? "FAILED" : "ok");
    return fail ? 1 : 0;
}
