// A reader of FASTA and FASTQ sequences, in batches for the GPU: the input side of the counter
// (counter/Fastx_Reader.hpp:13-52 in the reference). The first character sets the format, '>' for FASTA, '@' for
// FASTQ; a FASTA sequence joins its lines up to the next header; a FASTQ record is four lines, its quality line as
// long as its sequence. Lines end with "\n" or "\r\n". Regular files and pipes alike are read through one buffer,
// sequentially. Malformed input, gzip input and unreadable paths throw std::runtime_error.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace kache_b200
{

class Fastx_Reader
{
public:

    explicit Fastx_Reader(const std::string& path);
    ~Fastx_Reader();
    Fastx_Reader(const Fastx_Reader&) = delete;
    Fastx_Reader& operator=(const Fastx_Reader&) = delete;

    // Replaces `bases` and `lens` with the next non-empty sequences, concatenated, whole, until at least `max_bases`
    // bases are in (or the input ends). Returns false iff there were none left.
    bool next(std::vector<char>& bases, std::vector<size_t>& lens, size_t max_bases);

private:

    int fd_ = -1;
    std::string path_;
    std::vector<char> buf_;
    size_t at_ = 0, end_ = 0;
    bool eof_ = false;
    bool fastq_ = false;
    std::string line_;          // A line that crossed the buffer's end.
    bool have_header_ = false;  // FASTA: the next record's header was already read.

    bool fill();
    // Puts the next line, without its end, at [p, p + n); false at the end of the input.
    bool read_line(const char*& p, size_t& n);
    [[noreturn]] void malformed(const char* what) const;
};

}
