// FASTA / FASTQ batches for the counter; see fastx.hpp.
#include "fastx.hpp"

#include <cerrno>
#include <cstring>
#include <fcntl.h>
#include <stdexcept>
#include <unistd.h>

namespace kache_b200
{

Fastx_Reader::Fastx_Reader(const std::string& path): path_(path), buf_(size_t(8) << 20)
{
    fd_ = ::open(path.c_str(), O_RDONLY);
    if(fd_ < 0)
        throw std::runtime_error("cannot open " + path + ": " + std::strerror(errno));
    if(!fill())
        return; // Empty input: no sequences.
    const unsigned char c0 = static_cast<unsigned char>(buf_[at_]);
    if(c0 == 0x1f && (end_ - at_ < 2 || static_cast<unsigned char>(buf_[at_ + 1]) == 0x8b))
        throw std::runtime_error(path + " is gzip-compressed; decompress it, e.g. into a pipe");
    if(c0 != '>' && c0 != '@')
        throw std::runtime_error(path + " is neither FASTA nor FASTQ: it starts with neither '>' nor '@'");
    fastq_ = (c0 == '@');
}

Fastx_Reader::~Fastx_Reader()
{
    if(fd_ >= 0)
        ::close(fd_);
}

bool Fastx_Reader::fill()
{
    if(eof_)
        return at_ < end_;
    if(at_ > 0 && at_ < end_)
        std::memmove(buf_.data(), buf_.data() + at_, end_ - at_);
    end_ -= at_, at_ = 0;
    while(end_ < buf_.size())
    {
        const ssize_t r = ::read(fd_, buf_.data() + end_, buf_.size() - end_);
        if(r < 0)
        {
            if(errno == EINTR)
                continue;
            throw std::runtime_error("cannot read " + path_ + ": " + std::strerror(errno));
        }
        if(r == 0)
        {
            eof_ = true;
            break;
        }
        end_ += static_cast<size_t>(r);
    }
    return at_ < end_;
}

bool Fastx_Reader::read_line(const char*& p, size_t& n)
{
    line_.clear();
    while(true)
    {
        if(at_ == end_ && !fill())
        {
            if(line_.empty())
                return false;
            break;  // A last line without its end.
        }
        const char* s = buf_.data() + at_;
        const char* e = static_cast<const char*>(std::memchr(s, '\n', end_ - at_));
        if(e)
        {
            const size_t m = static_cast<size_t>(e - s);
            at_ += m + 1;
            if(line_.empty())
            {
                p = s, n = m;
                if(n && p[n - 1] == '\r')
                    n--;
                return true;
            }
            line_.append(s, m);
            break;
        }
        line_.append(s, end_ - at_);
        at_ = end_;
    }
    if(!line_.empty() && line_.back() == '\r')
        line_.pop_back();
    p = line_.data(), n = line_.size();
    return true;
}

void Fastx_Reader::malformed(const char* what) const
{
    throw std::runtime_error(std::string("malformed ") + (fastq_ ? "FASTQ" : "FASTA") + " input in " + path_ + ": " + what);
}

bool Fastx_Reader::next(std::vector<char>& bases, std::vector<size_t>& lens, const size_t max_bases)
{
    bases.clear(), lens.clear();
    const char* p;
    size_t n;
    while(bases.size() < max_bases)
    {
        if(fastq_)
        {
            if(!read_line(p, n))
                break;
            if(n == 0)
                continue;   // Blank lines between records.
            if(p[0] != '@')
                malformed("a record does not start with '@'");
            if(!read_line(p, n))
                malformed("a record ends after its header");
            const size_t b0 = bases.size(), len = n;
            bases.insert(bases.end(), p, p + n);
            if(!read_line(p, n) || n == 0 || p[0] != '+')
                malformed("a record's third line does not start with '+'");
            if(!read_line(p, n) || n != len)
                malformed("a quality line differs in length from its sequence");
            if(len)
                lens.push_back(len);
            else
                bases.resize(b0);
        }
        else
        {
            if(!have_header_)
            {
                if(!read_line(p, n))
                    break;
                if(n == 0)
                    continue;
                if(p[0] != '>')
                    malformed("a record does not start with '>'");
            }
            have_header_ = false;
            const size_t b0 = bases.size();
            bool more = false;
            while(read_line(p, n))
            {
                if(n && p[0] == '>')
                {
                    have_header_ = more = true;
                    break;
                }
                bases.insert(bases.end(), p, p + n);
            }
            if(bases.size() > b0)
                lens.push_back(bases.size() - b0);
            if(!more)
                break;
        }
    }
    return !lens.empty();
}

}
