// Host side of the B200 table: device memory, batch staging, the sizing and resize schedule, and the launches.
//
// One Engine<k, l, V> owns one table in HBM. Its operations are those of the reference's
// Streaming_Kmer_Hash_Table<k, true, V, l> (include/Streaming_Kmer_Hash_Table.hpp:624-745), with the value
// functions as device functors. The capacity follows the reference exactly: cap_for at construction, then one
// doubling wherever the reference's per-user flush schedule would resize (:2244-2286, :1447-1455, :1679-1680);
// that schedule depends only on the per-call counts of inserted keys, which the kernels return exactly. The GPU
// table itself resizes between launches: a call's batch is cut into chunks sized so the table stays below full,
// and after each chunk the table is rebuilt at the capacity the schedule has reached.
#pragma once

#include "device_misc.cuh"
#include "device_lanes.cuh"
#include "host_copy.hpp"
#include "seg_tuner.hpp"
#include "kache_b200.h"

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

// The object behind the C interface's opaque handle: a table of one (k, l, value width), behind virtual calls.
struct kache_table
{
    const uint32_t kmer_k, kmer_l, value_bytes;   // k, l and the values' width (0 in a set).
    std::mutex reg;                     // Serialises registrations.
    std::atomic<uint32_t> user_c{0};    // Registered users.
    mutable std::mutex work;            // Serialises the table's GPU work.

    kache_table(uint32_t k, uint32_t l, uint32_t vb): kmer_k(k), kmer_l(l), value_bytes(vb) {}
    virtual ~kache_table() = default;

    virtual void set_stream(cudaStream_t s) = 0;
    virtual uint64_t upsert(uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t init) = 0;
    // As upsert, also putting the keys each sequence inserted at per_seq[0..n) (host memory).
    virtual uint64_t upsert_split(uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t init, uint64_t* per_seq) = 0;
    virtual uint64_t upsert_oriented(uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t xf, uint64_t xr) = 0;
    virtual uint64_t update(const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x) = 0;
    virtual void lookup(const char* const* seqs, const size_t* lens, size_t n, uint8_t* found, void* values, uint8_t* fwd) = 0;
    virtual void seq_reduce(const char* const* seqs, const size_t* lens, size_t n, int mode, uint64_t m_fwd, uint64_t m_rev, uint64_t* out) = 0;
    virtual void describe(const char* const* seqs, const size_t* lens, size_t n, uint64_t* key, uint64_t* h, uint8_t* cs, uint8_t* fwd, uint8_t* valid) = 0;
    virtual uint64_t upsert_dev(uint32_t user, const uint8_t* b, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x, uint64_t init) = 0;
    virtual uint64_t upsert_oriented_dev(uint32_t user, const uint8_t* b, const uint64_t* off, uint64_t n, uint32_t op, uint64_t xf, uint64_t xr) = 0;
    virtual uint64_t update_dev(const uint8_t* b, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x) = 0;
    virtual void lookup_dev(const uint8_t* b, const uint64_t* off, uint64_t n, uint8_t* found, void* values, uint8_t* fwd) = 0;
    virtual void count_dev(const uint8_t* b, const uint64_t* off, uint64_t n, uint64_t* counts) = 0;
    virtual void run_dev_batches(uint32_t user, uint32_t kind, uint32_t op, uint64_t x, uint64_t y, kache_dev_batch* bs, size_t count) = 0;
    // A batch shape staged once (kache_b200_prepare_dev), and lookups of batches of that shape that only launch.
    virtual kache_prepared* prepare_dev(const uint64_t* off, uint64_t n) = 0;
    virtual void lookup_prepared(const kache_prepared& p, const uint8_t* b, uint8_t* found, void* values, uint8_t* fwd) = 0;
    virtual void count_prepared(const kache_prepared& p, const uint8_t* b, uint64_t* counts) = 0;
    virtual uint64_t epoch() = 0;
    virtual bool get(const char* kmer, uint64_t& value) = 0;
    virtual uint64_t size() const = 0;
    virtual uint64_t capacity() const = 0;
    virtual uint64_t reduce(uint32_t what, uint64_t mask) = 0;
    virtual void for_each(uint32_t shards, uint32_t shard, kache_keys_fn f, void* ctx) = 0;
    virtual void histogram(uint64_t max, uint64_t* h) = 0;
    virtual void get_stats(kache_stats& out) = 0;
    virtual void clear() = 0;
    // The table's device view and stream, for entry points that launch their own kernels on it.
    virtual kache_b200::Dev_Table device_table() const = 0;
    virtual cudaStream_t stream() const = 0;
    virtual void profile(bool on) = 0;
    virtual void profile_read(uint32_t kind, double& ms, uint64_t& launches) = 0;
    // Failure injection for tests: the bound of the kernels' waits for a racing insert's publication, and a claim of
    // the canonical k-mer `key`'s slot left unpublished, as by an inserter that never finishes. Returns whether a slot
    // was claimed (its primary bucket had room).
    virtual void testing_wait_polls(uint32_t polls) = 0;
    virtual bool testing_plant_claim(uint64_t key) = 0;
};

namespace kache_b200
{

// A CUDA failure: the C interface maps it to KACHE_EINTERNAL; failed allocations throw std::bad_alloc instead.
struct Cuda_Error : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

inline void check(const cudaError_t e, const char* what)
{
    if(e == cudaSuccess)
        return;
    if(e == cudaErrorMemoryAllocation)
    {
        (void)cudaGetLastError();
        throw std::bad_alloc();
    }
    throw Cuda_Error(std::string(what) + ": " + cudaGetErrorString(e));
}

std::atomic<uint64_t>& launches();

// Failure injection for tests: while nonnegative, the countdown of the library's device and page-locked allocations
// before one fails as out of memory (0: the next one); -1 when off.
std::atomic<int64_t>& alloc_fail_countdown();

// Fails the allocation about to be made if the injected countdown reaches it.
inline void alloc_gate()
{
    auto& c = alloc_fail_countdown();
    for(int64_t v = c.load(); v >= 0; )
        if(c.compare_exchange_weak(v, v - 1))
        {
            if(v == 0)
                throw std::bad_alloc();
            return;
        }
}

// ---- Sizing, as the reference's (include/Streaming_Kmer_Hash_Table.hpp:383, 800-804, 1004-1011) ----------------

inline uint64_t ceil_pow2(uint64_t x)
{
    uint64_t p = 1;
    while(p < x)
        p <<= 1;
    return p;
}

inline uint64_t cap_for(const uint64_t max_sz, const double lf, const bool pow2)
{
    uint64_t cap = std::max<uint64_t>(1, static_cast<uint64_t>(std::ceil(static_cast<double>(max_sz) / lf / B)));
    while(static_cast<uint64_t>(static_cast<double>(cap * B) * lf) <= max_sz)
        cap++;
    return pow2 ? ceil_pow2(cap) : cap;
}

inline bool fits(const uint64_t max_sz, const double lf, const bool pow2)
{
    return static_cast<double>(max_sz) / lf / B <= static_cast<double>(max_buckets) && cap_for(max_sz, lf, pow2) <= max_buckets;
}

inline uint64_t step_for(const uint64_t th) { return std::clamp<uint64_t>(th / (8 * 128), 1, 16384); }

// ---- Memory ----------------------------------------------------------------------------------------------------

struct Dev_Buf
{
    void* p = nullptr;
    size_t bytes = 0;

    Dev_Buf() = default;
    Dev_Buf(const Dev_Buf&) = delete;
    Dev_Buf& operator=(const Dev_Buf&) = delete;
    ~Dev_Buf() { release(); }

    void release()
    {
        if(p)
            cudaFree(p);
        p = nullptr, bytes = 0;
    }

    // Grows to at least n bytes; the contents are lost on growth.
    void ensure(const size_t n)
    {
        if(n <= bytes)
            return;
        release();
        alloc_gate();
        check(cudaMalloc(&p, std::max<size_t>(n, 256)), "cudaMalloc");
        bytes = std::max<size_t>(n, 256);
    }

    template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct Pinned_Buf
{
    void* p = nullptr;
    size_t bytes = 0;

    Pinned_Buf() = default;
    Pinned_Buf(const Pinned_Buf&) = delete;
    Pinned_Buf& operator=(const Pinned_Buf&) = delete;
    ~Pinned_Buf() { release(); }

    void release()
    {
        if(p)
            cudaDeviceSynchronize(), cudaFreeHost(p);   // No copy may still read or write it.
        p = nullptr, bytes = 0;
    }

    // Grows to at least n bytes, at least doubling (page-locking is slow: growing batches reallocate rarely); the
    // contents are lost on growth.
    void ensure(const size_t n)
    {
        if(n <= bytes)
            return;
        const size_t m = std::max<size_t>({n + n / 4, 2 * bytes, size_t(1) << 20});
        release();
        alloc_gate();
        check(cudaHostAlloc(&p, m, cudaHostAllocDefault), "cudaHostAlloc");
        bytes = m;
    }

    template <typename T> T* as(size_t byte_off = 0) const { return reinterpret_cast<T*>(static_cast<char*>(p) + byte_off); }
};

// A pool of host threads, started once, for the copies between callers' buffers and pinned staging memory.
class Host_Pool
{
    std::vector<std::thread> W_;
    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(size_t, size_t)>* job_ = nullptr;
    size_t n_ = 0, parts_ = 0, finished_ = 0;
    std::atomic<size_t> next_{0};
    uint64_t gen_ = 0;
    bool stop_ = false;

    void work_parts()
    {
        for(size_t p; (p = next_++) < parts_; )
        {
            (*job_)(n_ * p / parts_, n_ * (p + 1) / parts_);
            std::lock_guard<std::mutex> g(mu_);
            if(++finished_ == parts_)
                done_cv_.notify_all();
        }
    }

    Host_Pool()
    {
        const size_t t_c = std::min<size_t>(31, std::max(1u, std::thread::hardware_concurrency()) - 1);
        for(size_t t = 0; t < t_c; ++t)
            W_.emplace_back([this]()
            {
                uint64_t seen = 0;
                while(true)
                {
                    {
                        std::unique_lock<std::mutex> g(mu_);
                        cv_.wait(g, [&](){ return stop_ || gen_ != seen; });
                        if(stop_)
                            return;
                        seen = gen_;
                    }
                    work_parts();
                }
            });
    }

public:

    ~Host_Pool()
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for(auto& w : W_)
            w.join();
    }

    static Host_Pool& get()
    {
        static Host_Pool pool;
        return pool;
    }

    // Runs f(s, e) over [0, n) in parts of at least `min_part`, on the pool and this thread; returns when all ran.
    void run(const size_t n, const size_t min_part, const std::function<void(size_t, size_t)>& f)
    {
        const size_t parts = std::min<size_t>(4 * (W_.size() + 1), std::max<size_t>(1, n / std::max<size_t>(1, min_part)));
        if(parts <= 1 || W_.empty())
        {
            f(0, n);
            return;
        }
        std::lock_guard<std::mutex> run_g(run_mu_);
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &f, n_ = n, parts_ = parts, finished_ = 0, next_ = 0;
            gen_++;
        }
        cv_.notify_all();
        work_parts();
        std::unique_lock<std::mutex> g(mu_);
        done_cv_.wait(g, [&](){ return finished_ == parts_; });
    }
};

inline void parallel_for(const size_t n, const size_t min_per_thread, const std::function<void(size_t, size_t)>& f)
{
    Host_Pool::get().run(n, min_per_thread, f);
}

inline bool host_acgt(const char c)
{
    const char x = static_cast<char>(c | 0x20);
    return x == 'a' || x == 'c' || x == 'g' || x == 't';
}

// ---- The lane kernel's autotuner: seg_tuner.hpp ------------------------------------------------------------------

}

// A batch shape staged once: its offsets, each sequence's first position, and the list of its 512-position segments,
// all in device memory owned here, for lookups that launch without staging (kache_b200_lookup_prepared).
struct kache_prepared
{
    const kache_table* t = nullptr;     // The table that staged it.
    kache_b200::Dev_Buf off, pos_off, segs;
    uint64_t n = 0, nsegs = 0, total_pos = 0;
    uint32_t seg_len = 0;
};

namespace kache_b200
{

// ---- The engine --------------------------------------------------------------------------------------------------

enum Kind : uint32_t { K_UPSERT = 0, K_UPDATE = 1, K_LOOKUP = 2, K_REDUCE = 3, K_RESIZE = 4, K_OTHER = 5, K_KINDS = 6 };

template <int k, int l, typename V>
class Engine final : public kache_table
{
    static constexpr bool set_ = std::is_void_v<V>;
    typedef typename Val_Of<V>::type VT;    // The values' type; a placeholder in a set.
    static constexpr size_t slot_bytes = set_ ? 8 : 16;

    cudaStream_t own_ = nullptr, stream_ = nullptr;
    int sm_count_ = 148;
    Dev_Table epoch_T_{};   // The arrays epoch() last saw, and its count of changes.
    uint64_t epoch_ = 0;
    uint32_t wait_polls_ = default_wait_polls;

    // The table.
    Dev_Buf cs_, spill_, slots_, ov_, ctr_;
    Dev_Buf cs2_, spill2_, slots2_, ov2_;   // The previous table's arrays, kept for the next resize to build into.
    Dev_Table T_{};
    uint64_t ov_slots_ = 0;

    // The reference's sizing state (include/Streaming_Kmer_Hash_Table.hpp:81-86, 224-229).
    const double lf_;
    const uint64_t cap0_;
    uint64_t cap_, resize_th_, step_, approx_sz_ = 0, size_ = 0;
    uint64_t pending_[KACHE_MAX_USERS] = {};
    double novelty_ = 0.5;      // Keys inserted per position in the last upsert call.
    bool novelty_seen_ = false; // Whether an upsert call has measured it.

    // Batches.
    Pinned_Buf pin_, pin_ctr_, pin_out_;
    static constexpr int out_depth = 4;     // D2H pieces in flight ahead of the copy-out.
    cudaEvent_t ev_out_[out_depth] = {};
    static constexpr int out_pieces = 8;    // Pieces of a lookup whose outputs are copied while the next computes.
    cudaStream_t copy_stream_ = nullptr, in_stream_ = nullptr;
    cudaEvent_t ev_piece_[out_pieces] = {}, ev_in_[out_pieces] = {};
    cudaEvent_t ev_stage_ = nullptr, ev_bases_ = nullptr;

    void piece_events()
    {
        if(!ev_piece_[0])
            for(int c = 0; c < out_pieces; ++c)
                check(cudaEventCreateWithFlags(&ev_piece_[c], cudaEventDisableTiming), "event"),
                check(cudaEventCreateWithFlags(&ev_in_[c], cudaEventDisableTiming), "event");
    }

    // The copy streams beside the table's stream: input bases cross on in_stream_, outputs return on copy_stream_.
    void side_streams()
    {
        if(!copy_stream_)
            check(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        if(!in_stream_)
            check(cudaStreamCreateWithFlags(&in_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        if(!ev_stage_)
            check(cudaEventCreateWithFlags(&ev_stage_, cudaEventDisableTiming), "event"),
            check(cudaEventCreateWithFlags(&ev_bases_, cudaEventDisableTiming), "event");
    }
    Pinned_Buf pin_piece_;
    Dev_Buf dbatch_, dout_, dretry_a_, dretry_b_, dscan_, dtmp_;
    Dev_Buf dhost_;     // A page-locked host batch's bases and offsets, copied as they lie.
    Dev_Buf dmulti_;    // Several device batches run as one: their descriptors and the merged sequence list.
    Pinned_Buf pin_multi_;

    // Profiling.
    bool prof_ = false;
    struct Ev { cudaEvent_t a, b; uint32_t kind; };
    std::vector<Ev> ev_;
    // The autotuner, and the current call's choice and lane-kernel event pairs.
    Seg_Tuner tuner_;
    int tune_kind_ = -1, tune_cand_ = -1;
    uint32_t last_seg_len_[3] = {lane_seg_positions, lane_seg_positions, lane_seg_positions};   // Per tuned kind.
    uint64_t tune_pos_ = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tune_ev_;
    size_t tune_used_ = 0;
    double prof_ms_[K_KINDS] = {};
    uint64_t prof_n_[K_KINDS] = {};

    // Device counters: [0] inserted/present, [1] overflow keys, [2] retry flag + error word, [3..4] scratch.
    unsigned long long* ctr() const { return ctr_.as<unsigned long long>(); }

    struct Batch_Info
    {
        Dev_Batch b{};
        uint64_t total_pos = 0;
        // Listed on the device in sequence order: seg_off[q] (device) counts the segments of the sequences before q,
        // so a range of sequences is a range of segments and of output positions. Null where listed otherwise.
        const uint64_t* seg_off = nullptr;
        // Set where the bases are still in page-locked host memory here, laid end to end (staged with defer_bases).
        const char* host_bases = nullptr;
        // Set where the bases cross in two halves of sequences (ev_in_[0], ev_in_[1]): the table's stream waits for
        // the first before any launch, lane launches over segments from half_seg on wait for the second.
        bool in_halves = false;
        uint64_t half_seg = 0;
    };

    int grid_for(const uint64_t warps_needed, const int warps_per_block) const
    {
        const uint64_t blocks = (warps_needed + warps_per_block - 1) / warps_per_block;
        return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(blocks, uint64_t(sm_count_) * 16)));
    }

    template <typename F> void launch(const uint32_t kind, const F& f)
    {
        Ev e{};
        if(prof_)
        {
            check(cudaEventCreate(&e.a), "event"), check(cudaEventCreate(&e.b), "event");
            e.kind = kind;
            check(cudaEventRecord(e.a, stream_), "record");
        }
        f();
        check(cudaGetLastError(), "kernel launch");
        launches()++;
        if(prof_)
        {
            check(cudaEventRecord(e.b, stream_), "record");
            ev_.push_back(e);
        }
    }

    void sync() { check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize"); }

    // Reads the device counters [0, n).
    const unsigned long long* read_ctr(const int n)
    {
        check(cudaMemcpyAsync(pin_ctr_.p, ctr(), n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_), "D2H counters");
        sync();
        const auto* c = pin_ctr_.as<unsigned long long>();
        if(c[2] >> 32)
            throw Cuda_Error("a bounded device wait ran out");
        return c;
    }

    void alloc_table(Dev_Buf& cs, Dev_Buf& spill, Dev_Buf& slots, const uint64_t cap)
    {
        cs.ensure(cap * B), spill.ensure(cap * 32), slots.ensure(cap * B * slot_bytes);
        check(cudaMemsetAsync(cs.p, 0, cap * B, stream_), "memset");
        check(cudaMemsetAsync(spill.p, 0, cap * 32, stream_), "memset");
        check(cudaMemsetAsync(slots.p, 0, cap * B * slot_bytes, stream_), "memset");
    }

    static void swap_bufs(Dev_Buf& a, Dev_Buf& b) { std::swap(a.p, b.p), std::swap(a.bytes, b.bytes); }

    // Overflow capacity for n keys at load 0.8, a power of 2 (include/Concurrent_Hash_Table.hpp:157-172).
    static uint64_t ov_slots_for(const uint64_t n) { return ceil_pow2(static_cast<uint64_t>(std::ceil(static_cast<double>(n) / 0.8))); }

    void set_ov(Dev_Table& T, Dev_Buf& ov, const uint64_t slots)
    {
        ov.ensure(slots * 32);
        check(cudaMemsetAsync(ov.p, 0, slots * 32, stream_), "memset");
        T.ov = ov.as<unsigned long long>();
        T.ov_mask = slots - 1;
        T.ov_probe = static_cast<uint32_t>(std::min<uint64_t>(slots, 4096));
    }

    void bind(Dev_Table& T, Dev_Buf& cs, Dev_Buf& spill, Dev_Buf& slots, const uint64_t cap)
    {
        T.cs = cs.as<uint8_t>(), T.spill = spill.as<uint32_t>(), T.slots = slots.as<unsigned long long>(), T.cap = cap;
        T.ov_count = ctr() + 1;
        T.err = reinterpret_cast<unsigned int*>(ctr() + 2) + 1;
        T.wait_polls = wait_polls_;
    }

    // Doubles the overflow table.
    void grow_overflow()
    {
        Dev_Buf nov;
        Dev_Table T2 = T_;
        const uint64_t old = ov_slots_;
        set_ov(T2, nov, old * 2);
        launch(K_OTHER, [&](){ ov_move_kernel<<<grid_for(old / 32 + 1, 8), 256, 0, stream_>>>(T_.ov, old, T2); });
        std::swap(ov_.p, nov.p), std::swap(ov_.bytes, nov.bytes);
        T_ = T2, T_.ov = ov_.as<unsigned long long>();
        ov_slots_ = old * 2;
        sync();
    }

    // Rebuilds the table at `new_cap` buckets (include/Streaming_Kmer_Hash_Table.hpp:1474-1681, out of place).
    void resize(const uint64_t new_cap)
    {
        if(new_cap > max_buckets)
            throw std::runtime_error("the table would exceed the most buckets supported");
        const uint64_t old_cap = T_.cap;
        uint32_t d = 0;
        while((old_cap << d) < new_cap)
            d++;
        if((old_cap << d) != new_cap)
            throw std::logic_error("a resize multiplies the bucket count by a power of 2");
        // The new buckets are written whole by split_kernel: no clearing.
        Dev_Buf &cs = cs2_, &spill = spill2_, &slots = slots2_, &ov = ov2_;
        cs.ensure(new_cap * B), spill.ensure(new_cap * 32), slots.ensure(new_cap * B * slot_bytes);
        Dev_Table T2{};
        bind(T2, cs, spill, slots, new_cap);
        const uint64_t ov_keys = read_ctr(2)[1];
        uint64_t ov_slots = ov_slots_for(std::max<uint64_t>({1024, new_cap, static_cast<uint64_t>(ov_keys * 1.5)}));
        set_ov(T2, ov, ov_slots);
        // First phase: keys at their primary buckets move directly. Second phase: the others and the overflow
        // table's keys, marked in `dretry_a_`, go through the insertion chain. Every allocation comes before the
        // live table's state changes, so that a failed one leaves the table as it was.
        const uint64_t main_slots = old_cap * B, total = main_slots + ov_slots_;
        dretry_dirty_ = true;
        dretry_a_.ensure(total / 8 + 8), dretry_b_.ensure(total / 8 + 8);
        // The keys move, so the overflow count starts over.
        check(cudaMemsetAsync(ctr() + 1, 0, sizeof(unsigned long long), stream_), "memset");
        check(cudaMemsetAsync(dretry_a_.p, 0, main_slots / 8, stream_), "memset");
        // Every overflow slot is marked for the second phase, unless the overflow table holds no key.
        check(cudaMemsetAsync(dretry_a_.as<char>() + main_slots / 8, ov_keys ? 0xFF : 0, ov_slots_ / 8, stream_), "memset");
        unsigned int* retried = reinterpret_cast<unsigned int*>(ctr() + 2);
        check(cudaMemsetAsync(retried, 0, 4, stream_), "memset");
        check(cudaMemsetAsync(dretry_b_.p, 0, total / 8 + 8, stream_), "memset");
        launch(K_RESIZE, [&](){ split_kernel<k, l, set_><<<grid_for(old_cap, 8), 256, 0, stream_>>>(T_, T2, d, dretry_a_.as<unsigned int>()); });
        launch(K_RESIZE, [&](){ rest_kernel<k, l, set_><<<grid_for(total / 1024 + 1, 8), 256, 0, stream_>>>(T_, T2, dretry_a_.as<unsigned int>(), total, dretry_b_.as<unsigned int>(), retried); });
        std::swap(dretry_a_.p, dretry_b_.p), std::swap(dretry_a_.bytes, dretry_b_.bytes);
        while(static_cast<uint32_t>(read_ctr(3)[2]))
        {
            // The new overflow table filled up: double it, then retry the keys that found it full.
            Dev_Buf nov;
            Dev_Table T3 = T2;
            set_ov(T3, nov, ov_slots * 2);
            check(cudaMemsetAsync(ctr() + 1, 0, sizeof(unsigned long long), stream_), "memset");
            launch(K_RESIZE, [&](){ ov_move_kernel<<<grid_for(ov_slots / 32 + 1, 8), 256, 0, stream_>>>(T2.ov, ov_slots, T3); });
            const uint64_t moved = read_ctr(2)[1];
            (void)moved;
            std::swap(ov.p, nov.p), std::swap(ov.bytes, nov.bytes);
            T2 = T3, T2.ov = ov.as<unsigned long long>();
            ov_slots *= 2;
            // ov_move_kernel does not count: recount by the slots it filled.
            recount_overflow(T2, ov_slots);
            check(cudaMemsetAsync(dretry_b_.p, 0, total / 8 + 8, stream_), "memset");
            check(cudaMemsetAsync(retried, 0, 4, stream_), "memset");
            launch(K_RESIZE, [&](){ rest_kernel<k, l, set_><<<grid_for(total / 1024 + 1, 8), 256, 0, stream_>>>(T_, T2, dretry_a_.as<unsigned int>(), total, dretry_b_.as<unsigned int>(), retried); });
            std::swap(dretry_a_.p, dretry_b_.p), std::swap(dretry_a_.bytes, dretry_b_.bytes);
        }
        sync();
        std::swap(cs_.p, cs.p), std::swap(cs_.bytes, cs.bytes);
        std::swap(spill_.p, spill.p), std::swap(spill_.bytes, spill.bytes);
        std::swap(slots_.p, slots.p), std::swap(slots_.bytes, slots.bytes);
        std::swap(ov_.p, ov.p), std::swap(ov_.bytes, ov.bytes);
        bind(T_, cs_, spill_, slots_, new_cap);
        T_.ov = ov_.as<unsigned long long>(), T_.ov_mask = ov_slots - 1, T_.ov_probe = T2.ov_probe;
        ov_slots_ = ov_slots;
        dretry_dirty_ = true;
    }

    // Sets the overflow count to the occupied slots of T's overflow table.
    void recount_overflow(const Dev_Table& T, const uint64_t slots)
    {
        check(cudaMemsetAsync(ctr() + 1, 0, sizeof(unsigned long long), stream_), "memset");
        Dev_Table U = T;
        U.cap = 0;
        unsigned long long* out = ctr() + 3;
        check(cudaMemsetAsync(out, 0, 8, stream_), "memset");
        U.ov_mask = slots - 1;
        launch(K_OTHER, [&](){ reduce_kernel<true, uint8_t><<<grid_for(slots / 32 + 1, 8), 256, 0, stream_>>>(U, 0, 0, out, 0, nullptr); });
        check(cudaMemcpyAsync(ctr() + 1, out, 8, cudaMemcpyDeviceToDevice, stream_), "copy");
    }

    bool dretry_dirty_ = true;
    std::vector<uint64_t> seg_hist_;

    // ---- Batches ----

    // Stages a host batch: offsets, positions and segments computed here, bases gathered into pinned memory and copied
    // in pieces, each piece's H2D copy running while the next one is gathered.
    // Positions per segment: 512 for the warp kernel (16 rows per warp); for the lane kernel 64, or down to 16 in a
    // batch too small to give each of the GPU's threads 64 positions, so that small batches still spread over every
    // SM; eight times longer while a sequence would have more segments than a list entry indexes.
    uint32_t builtin_seg_len(const uint64_t total_pos) const
    {
        const uint64_t threads = uint64_t(sm_count_) * 2048;
        uint32_t s = lane_seg_positions;
        while(s > 16 && total_pos < uint64_t(s) * threads)
            s /= 2;
        return s;
    }

    // The lane segment length for this call: the autotuner's pick for the call's kind, once the batch's positions are
    // known (total_pos = ~0 while they are not).
    uint32_t first_seg_len(const bool lanes, const uint64_t total_pos)
    {
        if(!lanes)
            return seg_positions;
        if(tune_kind_ < 0)
            return builtin_seg_len(total_pos);
        if(total_pos == ~0ull)
            return last_seg_len_[tune_kind_];     // Before counting: likely the length this kind's last call used.
        tune_cand_ = tuner_.pick(tune_kind_, total_pos, builtin_seg_len(total_pos));
        tune_pos_ = total_pos;
        return last_seg_len_[tune_kind_] = Seg_Tuner::seg_len_of(tune_cand_);
    }

    // Starts a tuned call of `kind` (0 upsert, 1 update, 2 per-sequence reduction); finish_tune() records it.
    void begin_tune(const int kind) { tune_kind_ = kind, tune_cand_ = -1, tune_pos_ = 0, tune_used_ = 0; }

    // After the call's last sync: its lane kernels' time goes to the tuner.
    void finish_tune()
    {
        double ms = 0;
        for(size_t i = 0; i < tune_used_; ++i)
        {
            float t = 0;
            if(cudaEventElapsedTime(&t, tune_ev_[i].first, tune_ev_[i].second) == cudaSuccess)
                ms += t;
            else
                (void)cudaGetLastError();
        }
        if(tune_used_ > 0)
            tuner_.record(tune_kind_, tune_pos_, tune_cand_, ms);
        tune_kind_ = -1, tune_cand_ = -1, tune_used_ = 0;
    }

    uint32_t seg_len_for(const bool lanes, const uint64_t max_pos, const uint64_t total_pos)
    {
        uint64_t s = first_seg_len(lanes, total_pos);
        while((max_pos + s - 1) / s > max_seg_index + 1)
            s *= 8;
        return static_cast<uint32_t>(s);
    }

    // Stages a host batch. With `defer_bases` (a lookup in pieces), a batch laid end to end in page-locked memory is
    // listed from its offsets alone and its bases are left for the caller to copy (to bi.b.bases), piece by piece;
    // bi.host_bases is then set.
    // A host batch's totals, read once: bases, the longest sequence's and all sequences' positions, and whether the
    // sequences lie end to end. Large batches are summed over the host pool.
    struct Host_Scan
    {
        uint64_t bytes = 0, max_pos = 0, all_pos = 0;
        bool contiguous = true;
    };

    Host_Scan scan_host(const char* const* seqs, const size_t* lens, const size_t n) const
    {
        constexpr size_t part = size_t(1) << 15;
        const size_t parts = (n + part - 1) / part;
        std::vector<Host_Scan> r(std::max<size_t>(parts, 1));
        parallel_for(parts, 1, [&](const size_t s, const size_t e)
        {
            for(size_t j = s; j < e; ++j)
            {
                Host_Scan& h = r[j];
                for(size_t i = j * part, i1 = std::min(n, (j + 1) * part); i < i1; ++i)
                {
                    h.bytes += lens[i];
                    const uint64_t np = lens[i] >= size_t(k) ? lens[i] - k + 1 : 0;
                    h.max_pos = std::max<uint64_t>(h.max_pos, np), h.all_pos += np;
                    if(i + 1 < n && seqs[i] + lens[i] != seqs[i + 1])
                        h.contiguous = false;
                }
            }
        });
        Host_Scan t;
        for(const auto& h : r)
            t.bytes += h.bytes, t.max_pos = std::max(t.max_pos, h.max_pos), t.all_pos += h.all_pos, t.contiguous &= h.contiguous;
        return t;
    }

    Batch_Info stage_host(const char* const* seqs, const size_t* lens, const size_t n, const bool lanes, const bool defer_bases = false,
                          const Host_Scan* scanned = nullptr)
    {
        const Host_Scan hs = scanned ? *scanned : scan_host(seqs, lens, n);
        const uint64_t bytes = hs.bytes, max_pos = hs.max_pos, all_pos = hs.all_pos;
        const bool contiguous = hs.contiguous;
        // Sequences laid end to end in page-locked memory are copied to the device as they lie, with no gather, and
        // listed in segments there (stage_dev): the host only writes the offsets, in streaming stores (host_copy.hpp).
        const bool direct = n > 0 && bytes > 0 && contiguous && pinned(seqs[0]) && pinned(seqs[0] + bytes - 1);
        if(direct)
        {
            pin_.ensure((n + 1) * 8);
            uint64_t* off = pin_.as<uint64_t>();
            const char* base = seqs[0];
            parallel_for(n, 1 << 16, [&](const size_t s, const size_t e)
            {
                for(size_t i = s; i < e; ++i)
                    stream_u64(off + i, static_cast<uint64_t>(seqs[i] - base));
                stream_fence();
            });
            off[n] = bytes;
            const size_t o_off = (bytes + 64 + 15) / 16 * 16;
            dhost_.ensure(o_off + (n + 1) * 8);
            char* d = dhost_.as<char>();
            check(cudaMemsetAsync(d + bytes, 0, 64, stream_), "memset");
            check(cudaMemcpyAsync(d + o_off, off, (n + 1) * 8, cudaMemcpyHostToDevice, stream_), "H2D offsets");
            // The bases cross next, on the input stream, while the segments are listed here (host-to-device copies
            // share a copy engine, so they follow the offsets); the table's stream waits for them before its next
            // launch.
            // A large batch for the lane kernel crosses in two halves of sequences, so that its first launch need not
            // wait for the second half (two at most: a half of a 150 bp read set still fills the GPU's lanes).
            const bool halves = !defer_bases && lanes && n > small_stage_max && bytes >= (size_t(32) << 20);
            const uint64_t q_half = n / 2, b_half = halves ? off[q_half] : bytes;
            if(!defer_bases)
            {
                side_streams();
                piece_events();
                check(cudaEventRecord(ev_stage_, stream_), "event record");
                check(cudaStreamWaitEvent(in_stream_, ev_stage_, 0), "event wait");
                check(cudaMemcpyAsync(d, base, b_half, cudaMemcpyHostToDevice, in_stream_), "H2D batch");
                check(cudaEventRecord(ev_in_[0], in_stream_), "event record");
                if(bytes > b_half)
                    check(cudaMemcpyAsync(d + b_half, base + b_half, bytes - b_half, cudaMemcpyHostToDevice, in_stream_), "H2D batch");
                check(cudaEventRecord(ev_bases_, in_stream_), "event record");
            }
            Batch_Info bi = stage_dev(reinterpret_cast<const uint8_t*>(d), reinterpret_cast<const uint64_t*>(d + o_off), n, lanes);
            if(defer_bases)
            {
                bi.host_bases = base;
                return bi;
            }
            if(halves && bi.seg_off)
            {
                uint64_t* h = pin_ctr_.as<uint64_t>(56);
                check(cudaMemcpyAsync(h, bi.seg_off + q_half, 8, cudaMemcpyDeviceToHost, stream_), "D2H");
                sync();
                bi.half_seg = *h;
                bi.in_halves = bi.half_seg > 0 && bi.half_seg < bi.b.nsegs;
            }
            check(cudaStreamWaitEvent(stream_, bi.in_halves ? ev_in_[0] : ev_bases_, 0), "event wait");
            return bi;
        }
        if(n >= host_list_max)
            return stage_gathered(seqs, lens, n, bytes, lanes);
        const uint32_t seg_len = seg_len_for(lanes, max_pos, all_pos);
        uint64_t nsegs = 0;
        for(size_t i = 0; i < n; ++i)
        {
            const uint64_t p = lens[i] >= size_t(k) ? lens[i] - k + 1 : 0;
            nsegs += (p + seg_len - 1) / seg_len;
        }
        const size_t o_off = 0, o_pos = o_off + (n + 1) * 8, o_seg = o_pos + (n + 1) * 8, o_bases = o_seg + nsegs * 8;
        const size_t total = o_bases + bytes + 64;
        pin_.ensure(total);
        auto* off = pin_.as<uint64_t>(o_off);
        auto* pos_off = pin_.as<uint64_t>(o_pos);
        auto* segs = pin_.as<uint64_t>(o_seg);
        char* bases = pin_.as<char>(o_bases);
        // Segments listed longest first (a counting sort by length), so that the 32 lanes of a warp, which step as
        // long as their longest segment, get segments of similar lengths.
        seg_hist_.assign(seg_len + 1, 0);
        uint64_t b = 0, p = 0;
        for(size_t i = 0; i < n; ++i)
        {
            off[i] = b, pos_off[i] = p;
            const uint64_t np = lens[i] >= size_t(k) ? lens[i] - k + 1 : 0;
            if(np)
                seg_hist_[seg_len] += np / seg_len, seg_hist_[np % seg_len]++;
            b += lens[i], p += np;
        }
        off[n] = b, pos_off[n] = p;
        seg_hist_[0] = 0;
        for(uint64_t len = seg_len, at = 0; len > 0; --len)
        {
            const uint64_t c = seg_hist_[len];
            seg_hist_[len] = at, at += c;
        }
        for(size_t i = 0; i < n; ++i)
        {
            const uint64_t np = lens[i] >= size_t(k) ? lens[i] - k + 1 : 0;
            for(uint64_t s = 0; s * seg_len < np; ++s)
            {
                const uint64_t len = std::min<uint64_t>(np - s * seg_len, seg_len);
                segs[seg_hist_[len]++] = (uint64_t(i) << 24) | s;
            }
        }
        dbatch_.ensure(total);
        char* d = dbatch_.as<char>();
        check(cudaMemcpyAsync(d, pin_.p, o_bases, cudaMemcpyHostToDevice, stream_), "H2D batch");
        constexpr uint64_t piece = uint64_t(32) << 20;
        for(size_t i0 = 0; i0 < n; )
        {
            size_t i1 = i0;
            while(i1 < n && off[i1] - off[i0] < piece)
                i1++;
            parallel_for(i1 - i0, 2048, [&](const size_t s, const size_t e)
            {
                Stream_Writer w(bases + off[i0 + s]);
                for(size_t i = i0 + s; i < i0 + e; ++i)
                    w.put(seqs[i], lens[i]);
                w.finish();
            });
            check(cudaMemcpyAsync(d + o_bases + off[i0], bases + off[i0], off[i1] - off[i0], cudaMemcpyHostToDevice, stream_), "H2D batch");
            i0 = i1;
        }
        Batch_Info bi;
        bi.b = Dev_Batch{reinterpret_cast<const uint8_t*>(d + o_bases), reinterpret_cast<const uint64_t*>(d + o_off),
                         reinterpret_cast<const uint64_t*>(d + o_seg), reinterpret_cast<const uint64_t*>(d + o_pos), n, nsegs, seg_len};
        bi.total_pos = p;
        return bi;
    }

    // Pageable batches of many sequences: gathered end to end into page-locked memory in pieces, each piece's copy to
    // the device overlapping the next piece's gather, then listed on the device as a page-locked batch is. Listing a
    // million reads on the host (three passes and a counting sort) would take longer than the kernel that follows.
    static constexpr size_t host_list_max = 16384;

    Batch_Info stage_gathered(const char* const* seqs, const size_t* lens, const size_t n, const uint64_t bytes, const bool lanes)
    {
        const size_t o_hb = (n + 1) * 8;
        pin_.ensure(o_hb + bytes + 64);
        auto* off = pin_.as<uint64_t>();
        char* hb = pin_.as<char>(o_hb);
        uint64_t b = 0;
        for(size_t i = 0; i < n; ++i)
            off[i] = b, b += lens[i];
        off[n] = b;
        const size_t o_off = (bytes + 64 + 15) / 16 * 16;
        dhost_.ensure(o_off + (n + 1) * 8);
        char* d = dhost_.as<char>();
        check(cudaMemcpyAsync(d + o_off, off, (n + 1) * 8, cudaMemcpyHostToDevice, stream_), "H2D offsets");
        constexpr uint64_t piece = uint64_t(16) << 20;
        for(size_t i0 = 0; i0 < n; )
        {
            size_t i1 = i0;
            while(i1 < n && off[i1] - off[i0] < piece)
                i1++;
            parallel_for(i1 - i0, 2048, [&](const size_t s, const size_t e)
            {
                Stream_Writer w(hb + off[i0 + s]);
                for(size_t i = i0 + s; i < i0 + e; ++i)
                    w.put(seqs[i], lens[i]);
                w.finish();
            });
            if(off[i1] > off[i0])
                check(cudaMemcpyAsync(d + off[i0], hb + off[i0], off[i1] - off[i0], cudaMemcpyHostToDevice, stream_), "H2D batch");
            i0 = i1;
        }
        check(cudaMemsetAsync(d + bytes, 0, 64, stream_), "memset");
        return stage_dev(reinterpret_cast<const uint8_t*>(d), reinterpret_cast<const uint64_t*>(d + o_off), n, lanes);
    }

    // stage_dev for a batch of at most small_stage_max sequences: one block counts and sums, one kernel lists.
    Batch_Info stage_dev_small(const uint8_t* bases, const uint64_t* off, const uint64_t n, const bool lanes)
    {
        dtmp_.ensure(2 * (n + 1) * 8);
        uint64_t* pos_off = dtmp_.as<uint64_t>();
        uint64_t* seg_off = pos_off + (n + 1);
        unsigned long long* out = ctr() + 3;    // Three words: positions, segments, too long.
        uint64_t* h = pin_ctr_.as<uint64_t>(32);
        uint32_t seg_len = first_seg_len(lanes, ~0ull);
        bool sized = false;
        for(;;)
        {
            launch(K_OTHER, [&](){ stage_small_kernel<<<1, 1024, 0, stream_>>>(off, n, k, seg_len, pos_off, seg_off, out); });
            check(cudaMemcpyAsync(h, out, 24, cudaMemcpyDeviceToHost, stream_), "D2H");
            sync();
            if(h[2])
            {
                seg_len *= 8;   // A sequence has more segments than a list entry indexes.
                sized = true;
                continue;
            }
            if(!sized && lanes)
            {
                sized = true;
                const uint32_t want = first_seg_len(lanes, h[0]);
                if(want != seg_len)
                {
                    seg_len = want;
                    continue;
                }
            }
            break;
        }
        const uint64_t nsegs = h[1];
        dbatch_.ensure(nsegs * 8 + 8);
        if(nsegs > 0)
            launch(K_OTHER, [&](){ segs_kernel<<<grid_for((nsegs + 31) / 32, 8), 256, 0, stream_>>>(seg_off, n, nsegs, dbatch_.as<uint64_t>()); });
        Batch_Info bi;
        bi.b = Dev_Batch{bases, off, dbatch_.as<uint64_t>(), pos_off, n, nsegs, seg_len};
        bi.total_pos = h[0];
        bi.seg_off = seg_off;
        return bi;
    }

    // Prepares a batch already in device memory: positions and segments computed on the device.
    Batch_Info stage_dev(const uint8_t* bases, const uint64_t* off, const uint64_t n, const bool lanes)
    {
        if(n > 0 && n <= small_stage_max)
            return stage_dev_small(bases, off, n, lanes);
        const size_t o_npos = 0, o_nseg = o_npos + (n + 1) * 8, o_pos = o_nseg + (n + 1) * 8, o_sego = o_pos + (n + 1) * 8;
        const size_t head = o_sego + (n + 1) * 8;
        dtmp_.ensure(head);
        char* d = dtmp_.as<char>();
        auto* npos = reinterpret_cast<uint64_t*>(d + o_npos);
        auto* nseg = reinterpret_cast<uint64_t*>(d + o_nseg);
        auto* pos_off = reinterpret_cast<uint64_t*>(d + o_pos);
        auto* seg_off = reinterpret_cast<uint64_t*>(d + o_sego);
        unsigned int* too_long = reinterpret_cast<unsigned int*>(ctr() + 3);
        uint64_t* h = pin_ctr_.as<uint64_t>(32);
        uint32_t seg_len = first_seg_len(lanes, ~0ull);
        bool sized = false;     // Whether the lane segments were fitted to the batch's positions.
        for(;;)
        {
            check(cudaMemsetAsync(too_long, 0, 4, stream_), "memset");
            if(n > 0)
                launch(K_OTHER, [&](){ batch_counts_kernel<<<(n + 255) / 256, 256, 0, stream_>>>(off, n, k, seg_len, npos, nseg, too_long); });
            check(cudaMemsetAsync(pos_off, 0, 8, stream_), "memset");
            check(cudaMemsetAsync(seg_off, 0, 8, stream_), "memset");
            size_t tmp = 0;
            if(n > 0)
            {
                check(cub::DeviceScan::InclusiveSum(nullptr, tmp, npos, pos_off + 1, static_cast<int64_t>(n), stream_), "scan");
                dscan_.ensure(tmp);
                check(cub::DeviceScan::InclusiveSum(dscan_.p, tmp, npos, pos_off + 1, static_cast<int64_t>(n), stream_), "scan");
                check(cub::DeviceScan::InclusiveSum(dscan_.p, tmp, nseg, seg_off + 1, static_cast<int64_t>(n), stream_), "scan");
            }
            check(cudaMemcpyAsync(h, pos_off + n, 8, cudaMemcpyDeviceToHost, stream_), "D2H");
            check(cudaMemcpyAsync(h + 1, seg_off + n, 8, cudaMemcpyDeviceToHost, stream_), "D2H");
            check(cudaMemcpyAsync(h + 2, too_long, 4, cudaMemcpyDeviceToHost, stream_), "D2H");
            sync();
            if(static_cast<uint32_t>(h[2]))
            {
                seg_len *= 8;   // A sequence has more segments than a list entry indexes.
                sized = true;
                continue;
            }
            if(!sized && lanes)
            {
                sized = true;
                const uint32_t want = first_seg_len(lanes, h[0]);
                if(want != seg_len)
                {
                    seg_len = want;     // Count again with the segment length chosen for this batch's size.
                    continue;
                }
            }
            break;
        }
        const uint64_t total_pos = h[0], nsegs = h[1];
        dbatch_.ensure(nsegs * 8 + 8);
        if(nsegs > 0)
            launch(K_OTHER, [&](){ segs_kernel<<<grid_for((nsegs + 31) / 32, 8), 256, 0, stream_>>>(seg_off, n, nsegs, dbatch_.as<uint64_t>()); });
        Batch_Info bi;
        bi.b = Dev_Batch{bases, off, dbatch_.as<uint64_t>(), pos_off, n, nsegs, seg_len};
        bi.total_pos = total_pos;
        bi.seg_off = seg_off;
        return bi;
    }

    // Operations without per-position output (upsert, update, per-sequence reductions) run one lane per segment
    // (device_lanes.cuh): rolling descriptions, and lanes of a warp on different reads. Lookups and descriptions, whose
    // outputs are per position, run one warp per segment (device_stream.cuh), so that a row's 32 outputs are written
    // as one coalesced store.
    template <typename Vis> void stream_launch(const uint32_t kind, const Batch_Info& bi, const uint64_t sb, const uint64_t se, const Vis& vis, const bool per_position = false)
    {
        if(se <= sb)
            return;
        if(bi.in_halves && se > bi.half_seg)
        {
            // Segments before half_seg read the first half of the bases, which has crossed; the rest wait for the
            // second.
            if(per_position || sb >= bi.half_seg)
                check(cudaStreamWaitEvent(stream_, ev_bases_, 0), "event wait");
            else
            {
                lane_launch(kind, bi, sb, bi.half_seg, vis);
                check(cudaStreamWaitEvent(stream_, ev_bases_, 0), "event wait");
                lane_launch(kind, bi, bi.half_seg, se, vis);
                return;
            }
        }
        if(per_position)
        {
            launch(kind, [&](){ stream_kernel<k, l, Vis><<<grid_for(se - sb, stream_warps), 32 * stream_warps, 0, stream_>>>(bi.b, sb, se, vis); });
            return;
        }
        lane_launch(kind, bi, sb, se, vis);
    }

    template <typename Vis> void lane_launch(const uint32_t kind, const Batch_Info& bi, const uint64_t sb, const uint64_t se, const Vis& vis)
    {
        const bool timed = tune_kind_ >= 0 && tune_cand_ >= 0;
        const uint64_t per_sm = timed ? Seg_Tuner::blocks_of(tune_cand_) : Seg_Tuner::blocks[0];
        const uint64_t blocks = std::min<uint64_t>((se - sb + lane_block - 1) / lane_block, uint64_t(sm_count_) * per_sm);
        unsigned long long* next = ctr() + 7;     // The lane kernel's work counter.
        check(cudaMemsetAsync(next, 0, sizeof(unsigned long long), stream_), "memset");
        if(timed)
        {
            if(tune_used_ == tune_ev_.size())
            {
                std::pair<cudaEvent_t, cudaEvent_t> e{};
                check(cudaEventCreate(&e.first), "event"), check(cudaEventCreate(&e.second), "event");
                tune_ev_.push_back(e);
            }
            check(cudaEventRecord(tune_ev_[tune_used_].first, stream_), "record");
        }
        launch(kind, [&](){ lane_kernel<k, l, Vis><<<static_cast<unsigned>(blocks), lane_block, 0, stream_>>>(bi.b, sb, se, next, vis); });
        if(timed)
            check(cudaEventRecord(tune_ev_[tune_used_++].second, stream_), "record");
    }

    // The reference's per-user flush accounting over one call (include/Streaming_Kmer_Hash_Table.hpp:2248-2286,
    // 2511): fed the call's inserted keys chunk by chunk, it doubles the capacity where the reference would.
    // The schedule's state (approximate size, capacity in buckets, resize threshold, flush step), either the
    // engine's own or a copy for a prediction.
    struct Sched
    {
        uint64_t &approx, &cap, &th, &step;
        double lf;
    };

    struct Call_Acct
    {
        Sched S;
        uint64_t pending, flushed = 0, due, ins_c = 0;

        Call_Acct(const Sched& S, const uint64_t pending): S(S), pending(pending)
        {
            due = pending < S.step ? S.step - pending : 1;
        }

        void add(const uint64_t n)
        {
            const uint64_t end = ins_c + n;
            while(due <= end)
            {
                const uint64_t at = due;
                S.approx += pending + (at - flushed);
                pending = 0, flushed = at, due = at + S.step;
                if(S.approx >= S.th)
                {
                    if(2 * S.cap > max_buckets)
                        throw std::runtime_error("growing the table exceeds the most buckets supported");
                    S.cap *= 2;
                    S.th = static_cast<uint64_t>(static_cast<double>(S.cap * B) * S.lf);
                    S.step = step_for(S.th);
                }
            }
            ins_c = end;
        }

        // The user's keys inserted since its last flush, after the call.
        uint64_t left() const { return pending + (ins_c - flushed); }
    };

    // The capacity in buckets the schedule would reach if `user` inserted n more keys in one call.
    uint64_t predicted_cap(const uint32_t user, const uint64_t n) const
    {
        uint64_t a = approx_sz_, c = cap_, t = resize_th_, s = step_;
        Call_Acct sim(Sched{a, c, t, s, lf_}, pending_[user]);
        try
        {
            sim.add(n);
        }
        catch(const std::runtime_error&)
        {
        }
        return c;
    }

    // The bucket count to rebuild a non-empty table at when the schedule needs `target`: one doubling more while the
    // wider arrays take at most half the device memory free (counting the spare arrays a rebuild reuses), so that a
    // table growing call after call is rebuilt at every other doubling of its capacity, moving about a third fewer
    // keys over all its rebuilds (each of which rehashes every key it moves). Where keys sit is not observable; the
    // capacity reported stays the schedule's.
    uint64_t rebuild_cap(const uint64_t target)
    {
        const uint64_t wide = 2 * target;
        if(wide > max_buckets)
            return target;
        const size_t need = wide * (B + 32 + B * slot_bytes) + ov_slots_for(std::max<uint64_t>(1024, wide)) * 32;
        size_t free_b = 0, total_b = 0;
        check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
        const size_t spare = cs2_.bytes + spill2_.bytes + slots2_.bytes + ov2_.bytes;
        return 2 * need <= free_b + spare ? wide : target;
    }

    // Grows the device table to `target` buckets ahead of a call's inserts: where keys sit is not observable, so the
    // device table may have more buckets than the capacity the schedule reports, never fewer. An empty table is
    // reallocated and zeroed rather than rebuilt. Skipped if the arrays would not fit in free device memory.
    void grow_ahead(const uint64_t target)
    {
        if(target <= T_.cap)
            return;
        const uint64_t ov_slots = ov_slots_for(std::max<uint64_t>(1024, target));
        const size_t need = target * (B + 32 + B * slot_bytes) + ov_slots * 32;
        const bool allocated = size_ == 0 && cs_.bytes >= target * B && spill_.bytes >= target * 32 &&
                               slots_.bytes >= target * B * slot_bytes && ov_.bytes >= ov_slots * 32;
        if(!allocated)      // The arrays would be allocated: only if they fit in free device memory.
        {
            size_t free_b = 0, total_b = 0;
            check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
            const size_t held = size_ == 0 ? cs2_.bytes + spill2_.bytes + slots2_.bytes + ov2_.bytes : 0;
            if(need + (size_t(1) << 30) > free_b + held)
                return;
        }
        if(size_ != 0)
        {
            resize(rebuild_cap(target));
            return;
        }
        if(!allocated)
        {
            // Made in the spare arrays and swapped in, so that a failed allocation leaves the table as it was; the
            // arrays given up become the spares.
            alloc_table(cs2_, spill2_, slots2_, target);
            ov2_.ensure(ov_slots * 32);
            swap_bufs(cs_, cs2_), swap_bufs(spill_, spill2_), swap_bufs(slots_, slots2_), swap_bufs(ov_, ov2_);
        }
        else
        {
            check(cudaMemsetAsync(cs_.p, 0, target * B, stream_), "memset");
            check(cudaMemsetAsync(spill_.p, 0, target * 32, stream_), "memset");
            check(cudaMemsetAsync(slots_.p, 0, target * B * slot_bytes, stream_), "memset");
        }
        bind(T_, cs_, spill_, slots_, target);
        ov_slots_ = ov_slots;
        set_ov(T_, ov_, ov_slots_);
        check(cudaMemsetAsync(ctr() + 1, 0, sizeof(unsigned long long), stream_), "memset");
    }

    // Upserts a staged batch with the value functor `fn`, chunk by chunk (see the top of this file).
    template <typename Fn> uint64_t run_upsert(const uint32_t user, const Batch_Info& bi, const Fn& fn, unsigned long long* per_seq = nullptr)
    {
        const uint64_t nsegs = bi.b.nsegs;
        const double pos_per_seg = nsegs ? static_cast<double>(bi.total_pos) / nsegs : 1.0;
        uint64_t total_ins = 0;
        // Keys inserted per position: as the previous call measured (1/2 before the first), then as the last chunk
        // measured. The device table is first grown to the capacity the schedule would reach at that rate, so that
        // a call usually runs as one launch, with no rebuild. Before any call has measured it, the first chunk is
        // sized as if every position inserted a key, so that a table fed only new keys is never overfilled.
        double novelty = novelty_;
        bool assume_all_new = !novelty_seen_;
        grow_ahead(predicted_cap(user, static_cast<uint64_t>(novelty * static_cast<double>(bi.total_pos))));
        Call_Acct acct(Sched{approx_sz_, cap_, resize_th_, step_, lf_}, pending_[user]);
        const size_t bits = bi.total_pos / 8 + 8;
        unsigned int* retried = reinterpret_cast<unsigned int*>(ctr() + 2);

        for(uint64_t sb = 0; sb < nsegs; )
        {
            if(dretry_dirty_ || dretry_a_.bytes < bits || dretry_b_.bytes < bits)
            {
                dretry_a_.ensure(bits), dretry_b_.ensure(bits);
                check(cudaMemsetAsync(dretry_a_.p, 0, dretry_a_.bytes, stream_), "memset");
                dretry_dirty_ = false;
            }
            // A chunk may take the device table to 95 % of its slots, at a quarter above the expected rate (and at
            // least a quarter of the positions); the schedule then resizes it, as the reference would.
            const double slots = static_cast<double>(T_.cap * B);
            const double room = std::max(0.95 * slots - static_cast<double>(size_), 0.05 * slots);
            const double rate = assume_all_new ? 1.0 : std::max(1.25 * novelty, 0.25);
            const double want_pos = room / rate;
            uint64_t se = sb + std::max<uint64_t>(1, static_cast<uint64_t>(want_pos / pos_per_seg));
            // No small last chunk (it would run with too few lanes to fill the GPU), if the rest fits at the rate.
            if(se + (se - sb) / 2 >= nsegs && static_cast<double>(nsegs - sb) * pos_per_seg * rate <= 1.25 * room)
                se = nsegs;
            se = std::min(se, nsegs);
            assume_all_new = false;

            check(cudaMemsetAsync(ctr(), 0, 8, stream_), "memset");
            check(cudaMemsetAsync(retried, 0, 4, stream_), "memset");
            Upsert_Visitor<set_, VT, Fn> vis{T_, fn, bi.b.pos_off, ctr(), dretry_a_.as<unsigned int>(), nullptr, retried, 0, per_seq};
            stream_launch(K_UPSERT, bi, sb, se, vis);
            const unsigned long long* c = read_ctr(3);
            uint64_t ins = c[0];
            while(static_cast<uint32_t>(c[2]))
            {
                dretry_dirty_ = true;   // Until the retries end with no bit left set (a failure may come first).
                grow_overflow();
                check(cudaMemsetAsync(ctr(), 0, 8, stream_), "memset");
                check(cudaMemsetAsync(retried, 0, 4, stream_), "memset");
                check(cudaMemsetAsync(dretry_b_.p, 0, bits, stream_), "memset");
                Upsert_Visitor<set_, VT, Fn> rv{T_, fn, bi.b.pos_off, ctr(), dretry_b_.as<unsigned int>(), dretry_a_.as<unsigned int>(), retried, 0, per_seq};
                stream_launch(K_UPSERT, bi, sb, se, rv);
                check(cudaMemsetAsync(dretry_a_.p, 0, bits, stream_), "memset");
                std::swap(dretry_a_.p, dretry_b_.p), std::swap(dretry_a_.bytes, dretry_b_.bytes);
                c = read_ctr(3);
                ins += c[0];
            }

            const double chunk_pos = (se - sb) * pos_per_seg;
            novelty = chunk_pos > 0 ? std::max(static_cast<double>(ins) / chunk_pos, 1e-3) : novelty;
            size_ += ins, total_ins += ins;
            acct.add(ins);
            if(cap_ > T_.cap)
                resize(rebuild_cap(cap_));
            if(c[1] * 4 > ov_slots_ * 3)
                grow_overflow();
            sb = se;
        }
        pending_[user] = acct.left();
        if(bi.total_pos > 0)
            novelty_ = std::max(static_cast<double>(total_ins) / static_cast<double>(bi.total_pos), 1e-3), novelty_seen_ = true;
        return total_ins;
    }

    template <typename Fn> uint64_t run_update(const Batch_Info& bi, const Fn& fn)
    {
        check(cudaMemsetAsync(ctr(), 0, 8, stream_), "memset");
        Update_Visitor<VT, Fn> vis{T_, fn, ctr(), 0};
        stream_launch(K_UPDATE, bi, 0, bi.b.nsegs, vis);
        return read_ctr(3)[0];
    }

    void run_lookup(const Batch_Info& bi, uint8_t* found, VT* values, uint8_t* fwd)
    {
        Lookup_Visitor<set_, VT> vis{T_, bi.b.pos_off, found, values, fwd, 0};
        stream_launch(K_LOOKUP, bi, 0, bi.b.nsegs, vis, true);
    }

    void run_seq_reduce(const Batch_Info& bi, const int mode, const uint64_t mf, const uint64_t mr, unsigned long long* out)
    {
        check(cudaMemsetAsync(out, 0, bi.b.n * 8, stream_), "memset");
        if(mode == 0)
            stream_launch(K_REDUCE, bi, 0, bi.b.nsegs, Seq_Reduce_Visitor<set_, VT, 0>{T_, out, VT(mf), VT(mr), 0, 0});
        else if(mode == 1)
            stream_launch(K_REDUCE, bi, 0, bi.b.nsegs, Seq_Reduce_Visitor<set_, VT, 1>{T_, out, VT(mf), VT(mr), 0, 0});
        else
            stream_launch(K_REDUCE, bi, 0, bi.b.nsegs, Seq_Reduce_Visitor<set_, VT, 2>{T_, out, VT(mf), VT(mr), 0, 0});
    }

    // Whether host memory at p is page-locked (the caller's cudaHostAlloc'd or registered memory): copies then use it
    // directly.
    static bool pinned(const void* p)
    {
        if(p == nullptr)
            return false;
        cudaPointerAttributes a{};
        if(cudaPointerGetAttributes(&a, p) != cudaSuccess)
        {
            (void)cudaGetLastError();
            return false;
        }
        return a.type == cudaMemoryTypeHost;
    }

    // The device address of `bytes` of page-locked host memory at p (one allocation, mapped into the device's address
    // space, as cudaHostAlloc'd memory is on 64-bit systems), or null.
    static uint64_t host_bytes(const size_t* lens, const size_t n)
    {
        uint64_t b = 0;
        for(size_t i = 0; i < n; ++i)
            b += lens[i];
        return b;
    }

    bool pinned_range(const void* p, const size_t bytes) const
    {
        return p != nullptr && bytes > 0 && pinned(p) && pinned(static_cast<const char*>(p) + bytes - 1);
    }

    // A lookup in `out_pieces` pieces of sequences (a batch listed in sequence order), each piece's outputs copied to
    // page-locked host memory on the copy stream once the piece's kernel has run, while the next piece computes.
    void lookup_pieces(const Batch_Info& bi, uint8_t* d_found, VT* d_val, uint8_t* d_fwd, uint8_t* found, VT* values, uint8_t* fwd)
    {
        side_streams();
        piece_events();
        // Piece boundaries at sequences c * n / pieces: their first output position, first segment and first base.
        const uint64_t n = bi.b.n;
        pin_piece_.ensure(3 * (out_pieces + 1) * 8);
        auto* h = pin_piece_.as<uint64_t>();
        for(int c = 0; c <= out_pieces; ++c)
        {
            const uint64_t q = n * c / out_pieces;
            check(cudaMemcpyAsync(h + c, bi.b.pos_off + q, 8, cudaMemcpyDeviceToHost, stream_), "D2H");
            check(cudaMemcpyAsync(h + out_pieces + 1 + c, bi.seg_off + q, 8, cudaMemcpyDeviceToHost, stream_), "D2H");
            if(bi.host_bases)
                check(cudaMemcpyAsync(h + 2 * (out_pieces + 1) + c, bi.b.off + q, 8, cudaMemcpyDeviceToHost, stream_), "D2H");
        }
        sync();
        if(bi.host_bases)   // The input stream's copies come after this stream's earlier work.
            check(cudaEventRecord(ev_stage_, stream_), "event record"), check(cudaStreamWaitEvent(in_stream_, ev_stage_, 0), "event wait");
        Lookup_Visitor<set_, VT> vis{T_, bi.b.pos_off, d_found, d_val, d_fwd, 0};
        for(int c = 0; c < out_pieces; ++c)
        {
            const uint64_t p0 = h[c], p1 = h[c + 1], g0 = h[out_pieces + 1 + c], g1 = h[out_pieces + 2 + c];
            if(bi.host_bases)
            {
                // This piece's bases cross on the input stream while the previous piece computes.
                const uint64_t b0 = h[2 * (out_pieces + 1) + c], b1 = h[2 * (out_pieces + 1) + c + 1];
                if(b1 > b0)
                    check(cudaMemcpyAsync(const_cast<uint8_t*>(bi.b.bases) + b0, bi.host_bases + b0, b1 - b0, cudaMemcpyHostToDevice, in_stream_), "H2D batch");
                check(cudaEventRecord(ev_in_[c], in_stream_), "event record");
                check(cudaStreamWaitEvent(stream_, ev_in_[c], 0), "event wait");
            }
            stream_launch(K_LOOKUP, bi, g0, g1, vis, true);
            check(cudaEventRecord(ev_piece_[c], stream_), "event record");
            check(cudaStreamWaitEvent(copy_stream_, ev_piece_[c], 0), "event wait");
            if(p1 > p0)
            {
                check(cudaMemcpyAsync(found + p0, d_found + p0, p1 - p0, cudaMemcpyDeviceToHost, copy_stream_), "D2H");
                if(d_val)
                    check(cudaMemcpyAsync(values + p0, d_val + p0, (p1 - p0) * sizeof(VT), cudaMemcpyDeviceToHost, copy_stream_), "D2H");
                if(d_fwd)
                    check(cudaMemcpyAsync(fwd + p0, d_fwd + p0, p1 - p0, cudaMemcpyDeviceToHost, copy_stream_), "D2H");
            }
        }
        check(cudaStreamSynchronize(copy_stream_), "cudaStreamSynchronize");
        sync();
    }

    // Copies device output to a host buffer. Into page-locked memory, one copy. Into pageable memory, through pinned
    // pieces: up to `out_depth` D2H copies run ahead while the host pool copies finished pieces out.
    void d2h(void* dst, const void* src, const size_t bytes)
    {
        if(bytes == 0)
            return;
        if(pinned(dst) && pinned(static_cast<char*>(dst) + bytes - 1))
        {
            check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_), "D2H");
            sync();
            return;
        }
        constexpr size_t piece = size_t(32) << 20;
        pin_out_.ensure(out_depth * piece);
        if(!ev_out_[0])
            for(auto& e : ev_out_)
                check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        const size_t pieces = (bytes + piece - 1) / piece;
        const auto issue = [&](const size_t i)
        {
            const size_t o = i * piece, m = std::min(piece, bytes - o);
            check(cudaMemcpyAsync(pin_out_.as<char>((i % out_depth) * piece), static_cast<const char*>(src) + o, m, cudaMemcpyDeviceToHost, stream_), "D2H");
            check(cudaEventRecord(ev_out_[i % out_depth], stream_), "event record");
        };
        for(size_t i = 0; i < std::min<size_t>(out_depth, pieces); ++i)
            issue(i);
        for(size_t i = 0; i < pieces; ++i)
        {
            const size_t o = i * piece, m = std::min(piece, bytes - o);
            const char* stage = pin_out_.as<char>((i % out_depth) * piece);
            check(cudaEventSynchronize(ev_out_[i % out_depth]), "event sync");
            parallel_for(m, size_t(1) << 20, [&](const size_t s, const size_t e){ std::memcpy(static_cast<char*>(dst) + o + s, stage + s, e - s); });
            if(i + out_depth < pieces)
                issue(i + out_depth);
        }
    }

    static Op_Fn<VT> op_fn(const uint32_t op, const uint64_t x, const uint64_t init) { return Op_Fn<VT>{op, static_cast<VT>(x), static_cast<VT>(init)}; }

public:

    Engine(const uint64_t n, const double lf, const bool pow2):
          kache_table(k, l, set_ ? 0 : sizeof(VT))
        , lf_(lf)
        , cap0_(cap_for(n, lf, pow2))
        , cap_(cap0_)
    {
        if(cap_ > max_buckets)
            throw std::runtime_error("the table exceeds the most buckets supported");
        resize_th_ = static_cast<uint64_t>(static_cast<double>(cap_ * B) * lf_);
        step_ = step_for(resize_th_);
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        check(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, dev), "attribute");
        check(cudaStreamCreateWithFlags(&own_, cudaStreamNonBlocking), "cudaStreamCreate");
        stream_ = own_;
        pin_ctr_.ensure(64);
        ctr_.ensure(64);
        check(cudaMemsetAsync(ctr_.p, 0, 64, stream_), "memset");
        alloc_table(cs_, spill_, slots_, cap_);
        bind(T_, cs_, spill_, slots_, cap_);
        // The overflow table starts with room for max(1024, capacity / 32) keys (Streaming_Kmer_Hash_Table.hpp:775).
        ov_slots_ = ov_slots_for(std::max<uint64_t>(1024, cap_));
        set_ov(T_, ov_, ov_slots_);
        sync();
    }

    ~Engine() override
    {
        if(stream_)
            cudaStreamSynchronize(stream_);
        for(auto& e : ev_)
            cudaEventDestroy(e.a), cudaEventDestroy(e.b);
        for(auto& e : ev_out_)
            if(e)
                cudaEventDestroy(e);
        for(auto& e : tune_ev_)
            cudaEventDestroy(e.first), cudaEventDestroy(e.second);
        for(int c = 0; c < out_pieces; ++c)
        {
            if(ev_piece_[c])
                cudaEventDestroy(ev_piece_[c]);
            if(ev_in_[c])
                cudaEventDestroy(ev_in_[c]);
        }
        if(ev_stage_)
            cudaEventDestroy(ev_stage_), cudaEventDestroy(ev_bases_);
        if(copy_stream_)
            cudaStreamSynchronize(copy_stream_), cudaStreamDestroy(copy_stream_);
        if(in_stream_)
            cudaStreamSynchronize(in_stream_), cudaStreamDestroy(in_stream_);
        if(own_)
            cudaStreamDestroy(own_);
    }

    void set_stream(cudaStream_t s) override
    {
        std::lock_guard<std::mutex> g(work);
        sync();
        stream_ = s ? s : own_;
    }

    uint64_t upsert(uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t init) override
    {
        std::lock_guard<std::mutex> g(work);
        begin_tune(0);
        const auto bi = stage_host(seqs, lens, n, true);
        const uint64_t r = run_upsert(user, bi, op_fn(op, x, init));
        finish_tune();
        return r;
    }

    uint64_t upsert_split(uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t init, uint64_t* per_seq) override
    {
        std::lock_guard<std::mutex> g(work);
        begin_tune(0);
        const auto bi = stage_host(seqs, lens, n, true);
        dout_.ensure(n * 8 + 8);
        check(cudaMemsetAsync(dout_.p, 0, n * 8, stream_), "memset");
        const uint64_t r = run_upsert(user, bi, op_fn(op, x, init), dout_.as<unsigned long long>());
        d2h(per_seq, dout_.p, n * 8);
        finish_tune();
        return r;
    }

    uint64_t upsert_oriented(uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t xf, uint64_t xr) override
    {
        if constexpr(set_)
            return 0;
        else
        {
            std::lock_guard<std::mutex> g(work);
            begin_tune(0);
            const auto bi = stage_host(seqs, lens, n, true);
            const uint64_t r = run_upsert(user, bi, Oriented_Op_Fn<VT>{op, static_cast<VT>(xf), static_cast<VT>(xr)});
            finish_tune();
            return r;
        }
    }

    uint64_t update(const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x) override
    {
        if constexpr(set_)
            return 0;
        else
        {
            std::lock_guard<std::mutex> g(work);
            begin_tune(1);
            const auto bi = stage_host(seqs, lens, n, true);
            const uint64_t r = run_update(bi, op_fn(op, x, 0));
            finish_tune();
            return r;
        }
    }

    void lookup(const char* const* seqs, const size_t* lens, size_t n, uint8_t* found, void* values, uint8_t* fwd) override
    {
        std::lock_guard<std::mutex> g(work);
        // With outputs in page-locked memory the lookup may run in pieces (below); then the bases of a batch laid end
        // to end in page-locked memory are copied piece by piece as well.
        const Host_Scan hs = scan_host(seqs, lens, n);
        const uint64_t P_est = hs.all_pos;
        const size_t vb_est = (!set_ && values) ? sizeof(VT) : 0;
        const bool out_pinned = P_est > 0 && pinned_range(found, P_est) && (!vb_est || pinned_range(values, P_est * vb_est)) &&
                                (!fwd || pinned_range(fwd, P_est));
        const bool pieces = out_pinned && n >= 2 * out_pieces && P_est >= (uint64_t(1) << 22);
        const auto bi = stage_host(seqs, lens, n, false, pieces, &hs);
        const uint64_t P = bi.total_pos;
        const size_t vb = (!set_ && values) ? sizeof(VT) : 0;
        const size_t a_found = (P + 15) / 16 * 16, a_val = (P * vb + 15) / 16 * 16;
        dout_.ensure(a_found + a_val + P + 64);
        uint8_t* d_found = dout_.as<uint8_t>();
        VT* d_val = vb ? reinterpret_cast<VT*>(d_found + a_found) : nullptr;
        uint8_t* d_fwd = fwd ? d_found + a_found + a_val : nullptr;
        // Outputs in page-locked memory, of a batch listed in sequence order: the lookup runs in pieces of sequences,
        // each piece's outputs copied by DMA on a second stream while the next piece computes. (The kernel writing
        // them into mapped host memory itself was measured slower: its 32- and 256-byte stores reach about 33 GB/s
        // over PCIe, a copy about 55.)
        if(pieces && bi.seg_off)
        {
            lookup_pieces(bi, d_found, d_val, d_fwd, found, static_cast<VT*>(values), fwd);
            return;
        }
        if(bi.host_bases)   // Staged for pieces but not run in them: the bases cross whole first.
            check(cudaMemcpyAsync(const_cast<uint8_t*>(bi.b.bases), bi.host_bases, bi.b.off ? host_bytes(lens, n) : 0, cudaMemcpyHostToDevice, stream_), "H2D batch");
        run_lookup(bi, d_found, d_val, d_fwd);
        d2h(found, d_found, P);
        if(vb)
            d2h(values, d_val, P * vb);
        if(fwd)
            d2h(fwd, d_fwd, P);
    }

    void seq_reduce(const char* const* seqs, const size_t* lens, size_t n, int mode, uint64_t m_fwd, uint64_t m_rev, uint64_t* out) override
    {
        std::lock_guard<std::mutex> g(work);
        begin_tune(2);
        const auto bi = stage_host(seqs, lens, n, true);
        dout_.ensure(n * 8 + 8);
        run_seq_reduce(bi, mode, m_fwd, m_rev, dout_.as<unsigned long long>());
        d2h(out, dout_.p, n * 8);
        finish_tune();
    }

    void describe(const char* const* seqs, const size_t* lens, size_t n, uint64_t* key, uint64_t* h, uint8_t* cs, uint8_t* fwd, uint8_t* valid) override
    {
        std::lock_guard<std::mutex> g(work);
        const auto bi = stage_host(seqs, lens, n, false);
        const uint64_t P = bi.total_pos;
        dout_.ensure(P * 19 + 64);
        auto* dk = dout_.as<uint64_t>();
        auto* dh = dk + P;
        auto* dc = reinterpret_cast<uint8_t*>(dh + P);
        stream_launch(K_OTHER, bi, 0, bi.b.nsegs, Describe_Visitor{bi.b.pos_off, dk, dh, dc, dc + P, dc + 2 * P, false}, true);
        d2h(key, dk, P * 8), d2h(h, dh, P * 8), d2h(cs, dc, P), d2h(fwd, dc + P, P), d2h(valid, dc + 2 * P, P);
    }

    uint64_t upsert_dev(uint32_t user, const uint8_t* b, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x, uint64_t init) override
    {
        std::lock_guard<std::mutex> g(work);
        begin_tune(0);
        const auto bi = stage_dev(b, off, n, true);
        const uint64_t r = run_upsert(user, bi, op_fn(op, x, init));
        finish_tune();
        return r;
    }

    uint64_t upsert_oriented_dev(uint32_t user, const uint8_t* b, const uint64_t* off, uint64_t n, uint32_t op, uint64_t xf, uint64_t xr) override
    {
        if constexpr(set_)
            return 0;
        else
        {
            std::lock_guard<std::mutex> g(work);
            begin_tune(0);
            const auto bi = stage_dev(b, off, n, true);
            const uint64_t r = run_upsert(user, bi, Oriented_Op_Fn<VT>{op, static_cast<VT>(xf), static_cast<VT>(xr)});
            finish_tune();
            return r;
        }
    }

    uint64_t update_dev(const uint8_t* b, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x) override
    {
        if constexpr(set_)
            return 0;
        else
        {
            std::lock_guard<std::mutex> g(work);
            begin_tune(1);
            const auto bi = stage_dev(b, off, n, true);
            const uint64_t r = run_update(bi, op_fn(op, x, 0));
            finish_tune();
            return r;
        }
    }

    void lookup_dev(const uint8_t* b, const uint64_t* off, uint64_t n, uint8_t* found, void* values, uint8_t* fwd) override
    {
        std::lock_guard<std::mutex> g(work);
        const auto bi = stage_dev(b, off, n, false);
        run_lookup(bi, found, set_ ? nullptr : static_cast<VT*>(values), fwd);
        sync();
    }

    // Stages a batch shape once: the lookup's segment list and each sequence's first position, copied into the
    // handle, so that lookups of batches with these offsets need neither staging nor a sync.
    kache_prepared* prepare_dev(const uint64_t* off, const uint64_t n) override
    {
        std::lock_guard<std::mutex> g(work);
        const auto bi = stage_dev(nullptr, off, n, false);
        auto* p = new kache_prepared;
        try
        {
            p->t = this, p->n = n, p->nsegs = bi.b.nsegs, p->total_pos = bi.total_pos, p->seg_len = bi.b.seg_len;
            p->off.ensure((n + 1) * 8), p->pos_off.ensure((n + 1) * 8), p->segs.ensure(bi.b.nsegs * 8 + 8);
            if(n > 0)
            {
                check(cudaMemcpyAsync(p->off.p, off, (n + 1) * 8, cudaMemcpyDeviceToDevice, stream_), "copy");
                check(cudaMemcpyAsync(p->pos_off.p, bi.b.pos_off, (n + 1) * 8, cudaMemcpyDeviceToDevice, stream_), "copy");
            }
            if(bi.b.nsegs)
                check(cudaMemcpyAsync(p->segs.p, bi.b.segs, bi.b.nsegs * 8, cudaMemcpyDeviceToDevice, stream_), "copy");
            sync();
        }
        catch(...)
        {
            delete p;
            throw;
        }
        return p;
    }

    // A lookup of a batch of the prepared shape: one launch on the table's stream, no staging, no allocation, no
    // sync, so it can be captured in a CUDA graph. The launch takes the table's arrays as they are now.
    void lookup_prepared(const kache_prepared& p, const uint8_t* b, uint8_t* found, void* values, uint8_t* fwd) override
    {
        std::lock_guard<std::mutex> g(work);
        Batch_Info bi;
        bi.b = Dev_Batch{b, p.off.as<uint64_t>(), p.segs.as<uint64_t>(), p.pos_off.as<uint64_t>(), p.n, p.nsegs, p.seg_len};
        bi.total_pos = p.total_pos;
        run_lookup(bi, found, set_ ? nullptr : static_cast<VT*>(values), fwd);
    }

    // Per-sequence counts of present k-mers of a batch of the prepared shape: a memset and one launch of the warp
    // kernel (one atomic per segment), capturable as lookup_prepared is.
    void count_prepared(const kache_prepared& p, const uint8_t* b, uint64_t* counts) override
    {
        std::lock_guard<std::mutex> g(work);
        Batch_Info bi;
        bi.b = Dev_Batch{b, p.off.as<uint64_t>(), p.segs.as<uint64_t>(), p.pos_off.as<uint64_t>(), p.n, p.nsegs, p.seg_len};
        bi.total_pos = p.total_pos;
        auto* out = reinterpret_cast<unsigned long long*>(counts);
        if(p.n)
            check(cudaMemsetAsync(out, 0, p.n * 8, stream_), "memset");
        stream_launch(K_REDUCE, bi, 0, bi.b.nsegs, Seq_Reduce_Visitor<set_, VT, 0>{T_, out, VT(0), VT(0), 0, 0}, true);
    }

    // A number that stays the same while the table's device arrays do (a graph captured with a prepared lookup stays
    // valid), and changes when a call moved them (a rebuild, a clear, a larger overflow table).
    uint64_t epoch() override
    {
        std::lock_guard<std::mutex> g(work);
        const Dev_Table& a = epoch_T_;
        if(a.cs != T_.cs || a.spill != T_.spill || a.slots != T_.slots || a.cap != T_.cap || a.ov != T_.ov ||
           a.ov_mask != T_.ov_mask || a.ov_probe != T_.ov_probe || a.ov_count != T_.ov_count || a.err != T_.err)
            epoch_T_ = T_, ++epoch_;
        return epoch_;
    }

    void count_dev(const uint8_t* b, const uint64_t* off, uint64_t n, uint64_t* counts) override
    {
        std::lock_guard<std::mutex> g(work);
        begin_tune(2);
        const auto bi = stage_dev(b, off, n, true);
        run_seq_reduce(bi, 0, 0, 0, reinterpret_cast<unsigned long long*>(counts));
        sync();
        finish_tune();
    }

    // Several batches in device memory as one call: their sequences are listed as one batch whose lengths lie end to
    // end and whose sequences are read where they lie (Dev_Batch::seq_addr), so all share one segment list, one
    // launch and one pass of the resize schedule; results go back to each batch.
    void run_dev_batches(const uint32_t user, const uint32_t kind, const uint32_t op, const uint64_t x, const uint64_t y,
                         kache_dev_batch* const bs, const size_t count) override
    {
        std::lock_guard<std::mutex> g(work);
        uint64_t N = 0;
        for(size_t b = 0; b < count; ++b)
            bs[b].result = 0, N += bs[b].n;
        if(N == 0 || ((kind == KACHE_B200_RUN_UPSERT_ORIENTED || kind == KACHE_B200_RUN_UPDATE) && set_))
            return;
        // Descriptors, 8 words per batch; the merged list: offsets (N + 1), addresses (N), lengths (N), per-batch
        // first positions and results (count each), batch of each sequence (N, 32-bit).
        const size_t o_desc = 0, o_off = o_desc + count * 64, o_addr = o_off + (N + 1) * 8, o_len = o_addr + N * 8;
        const size_t o_pb = o_len + N * 8, o_res = o_pb + count * 8, o_bof = o_res + count * 8, total = o_bof + N * 4;
        pin_multi_.ensure(count * 64);
        auto* hd = pin_multi_.as<uint64_t>();
        for(size_t b = 0, s = 0; b < count; s += bs[b].n, ++b)
        {
            uint64_t* e = hd + 8 * b;
            e[0] = reinterpret_cast<uint64_t>(bs[b].d_bases), e[1] = reinterpret_cast<uint64_t>(bs[b].d_off);
            e[2] = bs[b].n, e[3] = s;
            e[4] = reinterpret_cast<uint64_t>(bs[b].out0), e[5] = reinterpret_cast<uint64_t>(bs[b].out1);
            e[6] = reinterpret_cast<uint64_t>(bs[b].out2), e[7] = 0;
        }
        dmulti_.ensure(total);
        char* d = dmulti_.as<char>();
        auto* desc = reinterpret_cast<uint64_t*>(d + o_desc);
        auto* voff = reinterpret_cast<uint64_t*>(d + o_off);
        auto* addr = reinterpret_cast<uint64_t*>(d + o_addr);
        auto* lens = reinterpret_cast<uint64_t*>(d + o_len);
        auto* pos_base = reinterpret_cast<uint64_t*>(d + o_pb);
        auto* res = reinterpret_cast<unsigned long long*>(d + o_res);
        auto* batch_of = reinterpret_cast<uint32_t*>(d + o_bof);
        check(cudaMemcpyAsync(desc, hd, count * 64, cudaMemcpyHostToDevice, stream_), "H2D descriptors");
        launch(K_OTHER, [&](){ batches_list_kernel<<<grid_for((N + 31) / 32, 8), 256, 0, stream_>>>(desc, count, N, lens, addr, batch_of); });
        check(cudaMemsetAsync(voff, 0, 8, stream_), "memset");
        size_t tmp = 0;
        check(cub::DeviceScan::InclusiveSum(nullptr, tmp, lens, voff + 1, static_cast<int64_t>(N), stream_), "scan");
        dscan_.ensure(tmp);
        check(cub::DeviceScan::InclusiveSum(dscan_.p, tmp, lens, voff + 1, static_cast<int64_t>(N), stream_), "scan");

        const bool lanes = kind != KACHE_B200_RUN_LOOKUP;
        if(kind == KACHE_B200_RUN_UPSERT || kind == KACHE_B200_RUN_UPSERT_ORIENTED)
            begin_tune(0);
        else if(kind == KACHE_B200_RUN_UPDATE)
            begin_tune(1);
        else if(kind == KACHE_B200_RUN_COUNT)
            begin_tune(2);
        auto bi = stage_dev(nullptr, voff, N, lanes);
        bi.b.seq_addr = addr;
        dout_.ensure(N * 8 + 8);
        auto* per_seq = dout_.as<unsigned long long>();
        check(cudaMemsetAsync(per_seq, 0, N * 8, stream_), "memset");
        if(kind == KACHE_B200_RUN_UPSERT)
            run_upsert(user, bi, op_fn(op, x, y), per_seq);
        else if(kind == KACHE_B200_RUN_UPSERT_ORIENTED)
        {
            if constexpr(!set_)
                run_upsert(user, bi, Oriented_Op_Fn<VT>{op, static_cast<VT>(x), static_cast<VT>(y)}, per_seq);
        }
        else if(kind == KACHE_B200_RUN_UPDATE)
        {
            if constexpr(!set_)
            {
                check(cudaMemsetAsync(ctr(), 0, 8, stream_), "memset");
                Update_Visitor<VT, Op_Fn<VT>> vis{T_, op_fn(op, x, 0), ctr(), 0};
                vis.per_seq = per_seq;
                stream_launch(K_UPDATE, bi, 0, bi.b.nsegs, vis);
            }
        }
        else if(kind == KACHE_B200_RUN_COUNT)
        {
            run_seq_reduce(bi, 0, 0, 0, per_seq);
            launch(K_OTHER, [&](){ batches_scatter_kernel<<<grid_for((N + 31) / 32, 8), 256, 0, stream_>>>(desc, per_seq, batch_of, N); });
        }
        else
        {
            launch(K_OTHER, [&](){ batches_pos_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream_>>>(desc, count, bi.b.pos_off, pos_base); });
            Lookup_Batches_Visitor<set_, VT> vis{{T_, bi.b.pos_off, nullptr, nullptr, nullptr, 0}, batch_of, desc, pos_base};
            stream_launch(K_LOOKUP, bi, 0, bi.b.nsegs, vis, true);
            launch(K_OTHER, [&](){ batches_hits_kernel<<<grid_for(N, 8), 256, 0, stream_>>>(desc, batch_of, bi.b.pos_off, pos_base, N, per_seq); });
        }
        // Per-batch results: the per-sequence counters (keys inserted, k-mers present, positions found, counts)
        // summed per batch.
        check(cudaMemsetAsync(res, 0, count * 8, stream_), "memset");
        launch(K_OTHER, [&](){ batches_sum_kernel<<<grid_for((N + 31) / 32 / 64 + 1, 8), 256, 0, stream_>>>(per_seq, batch_of, N, res); });
        auto* hr = pin_multi_.as<uint64_t>();
        check(cudaMemcpyAsync(hr, res, count * 8, cudaMemcpyDeviceToHost, stream_), "D2H results");
        sync();
        for(size_t b = 0; b < count; ++b)
            bs[b].result = hr[b];
        if(lanes)
            finish_tune();
    }

    bool get(const char* kmer, uint64_t& value) override
    {
        value = 0;
        uint64_t f = 0;
        for(int i = 0; i < k; ++i)
        {
            if(!host_acgt(kmer[i]))
                return false;
            f = (f << 2) | static_cast<uint64_t>(((kmer[i] >> 2) ^ (kmer[i] >> 1)) & 3);
        }
        uint64_t r = 0, y = f;
        for(int i = 0; i < k; ++i, y >>= 2)
            r = (r << 2) | (3 - (y & 3));
        const uint64_t key = f < r ? f : r;
        std::lock_guard<std::mutex> g(work);
        auto* h = pin_ctr_.as<uint64_t>(0);
        h[0] = key;
        unsigned long long* d = ctr() + 4;
        check(cudaMemcpyAsync(d, h, 8, cudaMemcpyHostToDevice, stream_), "H2D");
        launch(K_OTHER, [&](){ get_kernel<k, l, set_, VT><<<1, 32, 0, stream_>>>(T_, reinterpret_cast<const uint64_t*>(d), 1, d + 1); });
        check(cudaMemcpyAsync(h + 1, d + 1, 16, cudaMemcpyDeviceToHost, stream_), "D2H");
        sync();
        value = h[2];
        return h[1] != 0;
    }

    uint64_t size() const override { return size_; }
    uint64_t capacity() const override { return cap_ * B; }

    uint64_t reduce(uint32_t what, uint64_t mask) override
    {
        std::lock_guard<std::mutex> g(work);
        unsigned long long* out = ctr() + 3;
        check(cudaMemsetAsync(out, 0, 8, stream_), "memset");
        const uint64_t total = T_.cap * B + ov_slots_;
        launch(K_OTHER, [&](){ reduce_kernel<set_, VT><<<grid_for(total / 32 + 1, 8), 256, 0, stream_>>>(T_, what, mask, out, 0, nullptr); });
        return read_ctr(4)[3];
    }

    void histogram(uint64_t max, uint64_t* h) override
    {
        std::lock_guard<std::mutex> g(work);
        dout_.ensure((max + 1) * 8);
        check(cudaMemsetAsync(dout_.p, 0, (max + 1) * 8, stream_), "memset");
        const uint64_t total = T_.cap * B + ov_slots_;
        launch(K_OTHER, [&](){ reduce_kernel<set_, VT><<<grid_for(total / 32 + 1, 8), 256, 0, stream_>>>(T_, 3, 0, ctr() + 3, max, dout_.as<unsigned long long>()); });
        d2h(h, dout_.p, (max + 1) * 8);
        h[0] = 0;
    }

    void for_each(uint32_t shards, uint32_t shard, kache_keys_fn f, void* ctx) override
    {
        std::lock_guard<std::mutex> g(work);
        const uint64_t bb = T_.cap * shard / shards, be = T_.cap * (shard + 1) / shards;
        const uint64_t ov_range = (ov_slots_ + shards - 1) / shards;
        const uint64_t ob = std::min<uint64_t>(ov_range * shard, ov_slots_), oe = std::min<uint64_t>(ov_range * (shard + 1), ov_slots_);
        constexpr uint64_t piece = uint64_t(1) << 18;   // Buckets per device pass.
        constexpr size_t chunk = 4096;                  // Keys per callback (capi/Kmer_Table.hpp:234).
        std::vector<uint64_t> K, Vv;
        std::vector<VT> W(set_ ? 0 : chunk);
        bool done = false;
        const auto pass = [&](const uint64_t b0, const uint64_t b1, const uint64_t o0, const uint64_t o1)
        {
            const uint64_t slots = (b1 - b0) * B + (o1 - o0);
            if(slots == 0 || done)
                return;
            dout_.ensure(slots * 16 + 64);
            uint64_t* dk = dout_.as<uint64_t>();
            uint64_t* dv = set_ ? nullptr : dk + slots;
            unsigned long long* cnt = ctr() + 3;
            check(cudaMemsetAsync(cnt, 0, 8, stream_), "memset");
            launch(K_OTHER, [&](){ collect_kernel<set_><<<grid_for(slots / 32 + 1, 8), 256, 0, stream_>>>(T_, b0, b1, o0, o1, dk, dv, cnt); });
            const uint64_t m = read_ctr(4)[3];
            K.resize(m), Vv.resize(set_ ? 0 : m);
            d2h(K.data(), dk, m * 8);
            if(!set_)
                d2h(Vv.data(), dv, m * 8);
            for(uint64_t s = 0; s < m && !done; s += chunk)
            {
                const size_t c = std::min<uint64_t>(chunk, m - s);
                if constexpr(!set_)
                    for(size_t i = 0; i < c; ++i)
                        W[i] = static_cast<VT>(Vv[s + i]);
                done = f(ctx, K.data() + s, set_ ? nullptr : static_cast<const void*>(W.data()), c) != 0;
            }
        };
        for(uint64_t b = bb; b < be && !done; b += piece)
            pass(b, std::min(be, b + piece), 0, 0);
        for(uint64_t o = ob; o < oe && !done; o += piece * B)
            pass(0, 0, o, std::min(oe, o + piece * B));
    }

    void get_stats(kache_stats& out) override
    {
        std::lock_guard<std::mutex> g(work);
        out = kache_stats{};
        out.capacity = cap_ * B;
        out.bytes = T_.cap * (B + 32 + B * slot_bytes) + ov_slots_ * 32;
        out.keys = size_;
        unsigned long long* ps = ctr() + 3;
        check(cudaMemsetAsync(ps, 0, 16, stream_), "memset");
        launch(K_OTHER, [&](){ distribution_kernel<k, l, set_><<<grid_for(T_.cap * B / 32 + 1, 8), 256, 0, stream_>>>(T_, ps); });
        const auto* c = read_ctr(5);
        out.overflow_keys = c[1];
        const double p = static_cast<double>(c[3]), s = static_cast<double>(c[4]), o = static_cast<double>(c[1]);
        if(out.keys > 0)
        {
            const double t = p + s + o;
            out.primary_pct = p * 100.0 / t, out.secondary_pct = s * 100.0 / t, out.overflow_pct = o * 100.0 / t;
        }
    }

    // Upsert and update with any value functor (the C++ template facade's user functors: User_Fn,
    // User_Oriented_Fn), from a host batch.
    template <typename Fn> uint64_t upsert_with(const uint32_t user, const char* const* seqs, const size_t* lens, const size_t n, const Fn& fn)
    {
        std::lock_guard<std::mutex> g(work);
        begin_tune(0);
        const auto bi = stage_host(seqs, lens, n, true);
        const uint64_t r = run_upsert(user, bi, fn);
        finish_tune();
        return r;
    }

    template <typename Fn> uint64_t update_with(const char* const* seqs, const size_t* lens, const size_t n, const Fn& fn)
    {
        std::lock_guard<std::mutex> g(work);
        begin_tune(1);
        const auto bi = stage_host(seqs, lens, n, true);
        const uint64_t r = run_update(bi, fn);
        finish_tune();
        return r;
    }

    void testing_wait_polls(const uint32_t polls) override
    {
        std::lock_guard<std::mutex> g(work);
        wait_polls_ = polls;
        T_.wait_polls = polls;
    }

    bool testing_plant_claim(const uint64_t key) override
    {
        std::lock_guard<std::mutex> g(work);
        unsigned long long* d = ctr() + 4;
        launch(K_OTHER, [&](){ plant_claim_kernel<k, l, set_><<<1, 1, 0, stream_>>>(T_, key, d); });
        auto* h = pin_ctr_.as<uint64_t>(0);
        check(cudaMemcpyAsync(h, d, 8, cudaMemcpyDeviceToHost, stream_), "D2H");
        sync();
        return h[0] != 0;
    }

    Dev_Table device_table() const override { return T_; }
    cudaStream_t stream() const override { return stream_; }

    // Empties the table, back to its initial capacity and sizing state; registrations stay.
    void clear() override
    {
        std::lock_guard<std::mutex> g(work);
        if(T_.cap != cap0_)
        {
            alloc_table(cs_, spill_, slots_, cap0_);
            bind(T_, cs_, spill_, slots_, cap0_);
            ov_slots_ = ov_slots_for(std::max<uint64_t>(1024, cap0_));
            set_ov(T_, ov_, ov_slots_);
        }
        else
        {
            check(cudaMemsetAsync(cs_.p, 0, cap0_ * B, stream_), "memset");
            check(cudaMemsetAsync(spill_.p, 0, cap0_ * 32, stream_), "memset");
            check(cudaMemsetAsync(slots_.p, 0, cap0_ * B * slot_bytes, stream_), "memset");
            check(cudaMemsetAsync(ov_.p, 0, ov_slots_ * 32, stream_), "memset");
        }
        check(cudaMemsetAsync(ctr(), 0, 64, stream_), "memset");
        cap_ = cap0_;
        resize_th_ = static_cast<uint64_t>(static_cast<double>(cap_ * B) * lf_);
        step_ = step_for(resize_th_);
        approx_sz_ = 0, size_ = 0;
        std::fill(pending_, pending_ + KACHE_MAX_USERS, 0);
    }

    void profile(bool on) override
    {
        std::lock_guard<std::mutex> g(work);
        sync();
        for(auto& e : ev_)
            cudaEventDestroy(e.a), cudaEventDestroy(e.b);
        ev_.clear();
        std::fill(prof_ms_, prof_ms_ + K_KINDS, 0.0), std::fill(prof_n_, prof_n_ + K_KINDS, 0);
        prof_ = on;
    }

    void profile_read(uint32_t kind, double& ms, uint64_t& n) override
    {
        std::lock_guard<std::mutex> g(work);
        sync();
        for(auto& e : ev_)
        {
            float t = 0;
            check(cudaEventElapsedTime(&t, e.a, e.b), "elapsed");
            prof_ms_[e.kind] += t, prof_n_[e.kind]++;
            cudaEventDestroy(e.a), cudaEventDestroy(e.b);
        }
        ev_.clear();
        ms = kind < K_KINDS ? prof_ms_[kind] : 0, n = kind < K_KINDS ? prof_n_[kind] : 0;
    }
};

}
