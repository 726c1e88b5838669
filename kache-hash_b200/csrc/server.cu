// A request server over one table: callers submit upsert, lookup and count requests from any thread as they arrive;
// one dispatcher thread runs them on the GPU, merging the requests that are waiting when the GPU frees up into one
// launch (continuous batching): the oldest waiting request and every other waiting request of its kind (and, for
// upserts, its operation) become a single call over all their sequences, and each request gets its own share of the
// results back. Requests of one kind run in the order they were submitted; waiting requests of different kinds are
// concurrent, as the reference's users are, and a caller that needs one to see another waits for the first before
// submitting the second. Runs of different kinds never overlap, which keeps the reference's rule that queries do not
// overlap inserts
// (include/Streaming_Kmer_Hash_Table.hpp:2264-2266, capi/kache_capi.h:16-21); a resize an upsert run triggers happens
// inside its call, after the queries before it finished. A run is admitted only while its staging fits the byte budget
// (device memory for the merged batch), so a burst of requests waits rather than exhausting HBM. Two threads share the
// work: a stager forms the next run and gathers its reads end to end into one of two page-locked buffers while an
// executor runs the run before it on the GPU and copies its results out, so the host's copying overlaps the device.
// Requests whose reads and outputs are already in device memory (kache_b200_server_submit_dev) merge with each other
// into one call of the several-batches form (kache_b200_run_dev_batches): nothing to gather, nothing to copy out.
#include "engine.cuh"
#include "kache_b200.h"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace
{

using clock_type = std::chrono::steady_clock;

struct Request
{
    uint64_t ticket;
    uint32_t kind;                  // KACHE_B200_REQ_*
    std::vector<const char*> seqs;  // The caller's sequences: they stay the caller's and must outlive the request.
    std::vector<size_t> lens;
    uint32_t op;
    uint64_t x, init;
    void* out0;                     // lookup: found; count: counts
    void* out1;                     // lookup: values (or null)
    void* out2;                     // lookup: fwd (or null)
    // A device request (kache_b200_server_submit_dev): its n sequences are d_bases[d_off[i], d_off[i + 1]) and its
    // outputs out0..2 are device arrays; seqs and lens stay empty.
    bool dev = false;
    const uint8_t* d_bases = nullptr;
    const uint64_t* d_off = nullptr;
    uint64_t n_dev = 0;
    uint64_t positions = 0, bytes = 0, result = 0;
    int status = KACHE_OK;
    bool done = false;
    clock_type::time_point t_submit, t_done;
};

// A run ready for the GPU: its requests, and their sequences as the table is handed them -- gathered end to end into
// one of the page-locked staging buffers (slot 0 or 1; the table then copies them to the device as they lie and
// lists them there), or the callers' own memory (slot -1) for a run too large to stage.
struct Staged
{
    std::vector<Request*> g;
    int slot = -1;
    std::vector<const char*> seqs;
    std::vector<size_t> lens;
    std::vector<size_t> first;          // Each request's first sequence in the run.
    std::vector<uint64_t> pos_first;    // Each request's first k-mer position in the run.
};

}

struct kache_server
{
    kache_table* t;
    uint32_t user;
    uint64_t budget;                // Most staging bytes of one merged run.
    // Most k-mer positions of one merged run (unless its first request alone has more): enough to keep every SM
    // busy, few enough that a run's staging buffers stay reused and a request waits behind one run at most this big.
    static constexpr uint64_t run_positions = uint64_t(1) << 24;
    // Most sequences of one run of device requests (unless its first request alone has more). Their lengths lie in
    // device memory, unread by the host; they stage nothing on the host, so a run costs only its fixed per-call steps,
    // and fewer, larger runs keep the GPU busier: 2^20 short reads take a few milliseconds.
    static constexpr uint64_t dev_run_seqs = uint64_t(1) << 20;
    // Most bases of a run gathered into a staging buffer; larger runs are handed over from the callers' memory.
    static constexpr uint64_t stage_max = uint64_t(256) << 20;
    std::mutex mu;
    std::condition_variable cv, done_cv, ready_cv;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, Request*> all;
    uint64_t next_ticket = 1;
    bool stop = false;
    // Two threads: the stager forms runs and gathers their reads into a free staging buffer while the executor runs
    // the run before on the GPU, so the host's copying overlaps the device's work.
    std::thread worker, executor;
    kache_b200::Pinned_Buf stage[2];
    bool slot_busy[2] = {false, false};
    std::deque<Staged*> ready;
    bool staging_done = false;
    // Merged outputs, reused across runs, in page-locked memory (the table copies into it directly).
    kache_b200::Pinned_Buf found, fwd, values, counts;
    uint64_t runs = 0, merged = 0;

    void loop();
    void execute();
    void gather(Staged& st);
    void run(Staged& st);
};

namespace
{

// Device bytes a request's staging takes: bases, offsets, segment list and per-position outputs.
uint64_t request_bytes(const Request& r, const uint32_t k, const uint32_t vb)
{
    uint64_t bases = 0, pos = 0;
    for(const size_t len : r.lens)
        bases += len, pos += len >= k ? len - k + 1 : 0;
    const uint64_t per_pos = r.kind == KACHE_B200_REQ_LOOKUP ? 2 + vb : 1;
    return bases + 24 * r.lens.size() + pos * per_pos;
}

bool compatible(const Request& a, const Request& b)
{
    if(a.kind != b.kind || a.dev != b.dev)
        return false;
    if(a.kind == KACHE_B200_REQ_UPSERT)
        return a.op == b.op && a.x == b.x && a.init == b.init;
    if(a.kind == KACHE_B200_REQ_LOOKUP && !a.dev)     // Device lookups bind their own output arrays per request.
        return (a.out1 == nullptr) == (b.out1 == nullptr) && (a.out2 == nullptr) == (b.out2 == nullptr);
    return true;
}

}

void kache_server::loop()
{
    for(;;)
    {
        std::vector<Request*> g;
        {
            std::unique_lock<std::mutex> lk(mu);
            // The next run is formed once the executor has taken the one before it, so requests arriving meanwhile
            // merge into it instead of queueing as runs of their own.
            cv.wait(lk, [&](){ return stop || (!queue.empty() && ready.empty()); });
            if(queue.empty())
            {
                staging_done = true;
                lk.unlock();
                ready_cv.notify_all();
                return;
            }
            // The run: the head, then every waiting request that can merge with it, in arrival order, within budget;
            // the others keep their order in the queue.
            uint64_t bytes = 0, pos = 0, seqs = 0;
            std::deque<Request*> rest;
            for(Request* r : queue)
                if(g.empty() || (compatible(*r, *g.front()) && bytes + r->bytes <= budget &&
                                 (r->dev ? seqs + r->n_dev <= dev_run_seqs : pos + r->positions <= run_positions)))
                    bytes += r->bytes, pos += r->positions, seqs += r->n_dev, g.push_back(r);
                else
                    rest.push_back(r);
            queue.swap(rest);
        }
        auto* st = new Staged;
        st->g = std::move(g);
        gather(*st);
        {
            std::lock_guard<std::mutex> lk(mu);
            ready.push_back(st);
        }
        ready_cv.notify_all();
    }
}

// The stager's half of a run: lists its sequences and, unless it is too large, gathers them end to end into a free
// staging buffer (waiting for the executor to release one).
void kache_server::gather(Staged& st)
{
    const auto& g = st.g;
    if(g.front()->dev)
        return;     // Device requests are read where they lie.
    st.first.assign(g.size() + 1, 0), st.pos_first.assign(g.size() + 1, 0);
    uint64_t bytes = 0;
    for(size_t i = 0; i < g.size(); ++i)
    {
        st.lens.insert(st.lens.end(), g[i]->lens.begin(), g[i]->lens.end());
        st.first[i + 1] = st.lens.size();
        st.pos_first[i + 1] = st.pos_first[i] + g[i]->positions;
    }
    for(const size_t len : st.lens)
        bytes += len;
    const size_t n = st.lens.size();
    if(bytes > stage_max)
    {
        for(const Request* r : g)
            st.seqs.insert(st.seqs.end(), r->seqs.begin(), r->seqs.end());
        return;
    }
    {
        std::unique_lock<std::mutex> lk(mu);
        ready_cv.wait(lk, [&](){ return !slot_busy[0] || !slot_busy[1]; });
        st.slot = slot_busy[0] ? 1 : 0;
        slot_busy[st.slot] = true;
    }
    kache_b200::Pinned_Buf& buf = stage[st.slot];
    buf.ensure(bytes + 64);
    char* base = buf.as<char>();
    std::vector<uint64_t> off(n + 1, 0);
    for(size_t q = 0; q < n; ++q)
        off[q + 1] = off[q] + st.lens[q];
    st.seqs.resize(n);
    std::vector<const char*> src;
    src.reserve(n);
    for(const Request* r : g)
        src.insert(src.end(), r->seqs.begin(), r->seqs.end());
    // Streaming stores: the copy engine reads the staged bases next (host_copy.hpp).
    kache_b200::parallel_for(n, 2048, [&](const size_t s, const size_t e)
    {
        kache_b200::Stream_Writer w(base + off[s]);
        for(size_t q = s; q < e; ++q)
        {
            st.seqs[q] = base + off[q];
            w.put(src[q], st.lens[q]);
        }
        w.finish();
    });
}

// The executor: runs the staged runs on the GPU in the order they were formed.
void kache_server::execute()
{
    for(;;)
    {
        Staged* st = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            ready_cv.wait(lk, [&](){ return staging_done || !ready.empty(); });
            if(ready.empty())
                return;
            st = ready.front();
            ready.pop_front();
        }
        cv.notify_all();    // The stager may form the next run.
        run(*st);
        {
            std::lock_guard<std::mutex> lk(mu);
            const auto now = clock_type::now();
            for(Request* r : st->g)
                r->done = true, r->t_done = now;
            runs++, merged += st->g.size();
            if(st->slot >= 0)
                slot_busy[st->slot] = false;
        }
        done_cv.notify_all();
        ready_cv.notify_all();
        delete st;
    }
}

void kache_server::run(Staged& st)
{
    const auto& g = st.g;
    const auto& seqs = st.seqs;
    const auto& lens = st.lens;
    const auto& first = st.first;
    const auto& pos_first = st.pos_first;
    const size_t n = seqs.size();
    const Request& h = *g.front();
    const size_t vb = t->value_bytes;
    try
    {
        if(h.dev)
        {
            // One call of the several-batches form over the requests' device batches; each request's outputs go
            // straight to its own device arrays and its result comes back per batch.
            std::vector<kache_dev_batch> bs(g.size());
            for(size_t i = 0; i < g.size(); ++i)
                bs[i] = kache_dev_batch{g[i]->d_bases, g[i]->d_off, g[i]->n_dev, g[i]->out0, g[i]->out1, g[i]->out2, 0};
            const uint32_t kind = h.kind == KACHE_B200_REQ_UPSERT ? KACHE_B200_RUN_UPSERT
                                : h.kind == KACHE_B200_REQ_LOOKUP ? KACHE_B200_RUN_LOOKUP : KACHE_B200_RUN_COUNT;
            t->run_dev_batches(user, kind, h.op, h.x, h.init, bs.data(), bs.size());
            for(size_t i = 0; i < g.size(); ++i)
                g[i]->result = bs[i].result;
        }
        else if(h.kind == KACHE_B200_REQ_UPSERT)
        {
            counts.ensure((n + 1) * 8);
            const uint64_t* c = counts.as<uint64_t>();
            t->upsert_split(user, seqs.data(), lens.data(), n, h.op, h.x, h.init, counts.as<uint64_t>());
            for(size_t i = 0; i < g.size(); ++i)
            {
                uint64_t s = 0;
                for(size_t q = first[i]; q < first[i + 1]; ++q)
                    s += c[q];
                g[i]->result = s;
            }
        }
        else if(h.kind == KACHE_B200_REQ_LOOKUP)
        {
            const uint64_t P = pos_first.back();
            found.ensure(P + 16), fwd.ensure(h.out2 ? P + 16 : 16), values.ensure(h.out1 && vb ? P * vb + 16 : 16);
            const uint8_t* f = found.as<uint8_t>();
            const uint8_t* vals = values.as<uint8_t>();
            t->lookup(seqs.data(), lens.data(), n, found.as<uint8_t>(), h.out1 && vb ? values.p : nullptr, h.out2 ? fwd.as<uint8_t>() : nullptr);
            // Each request's share of the merged outputs to its own arrays, and its present positions: in parts of the
            // merged positions on the host pool's threads, a part spanning the requests it overlaps.
            std::vector<std::atomic<uint64_t>> hits(g.size());
            const uint8_t* fw = fwd.as<uint8_t>();
            kache_b200::parallel_for(P, size_t(1) << 20, [&](const size_t s, const size_t e)
            {
                size_t i = static_cast<size_t>(std::upper_bound(pos_first.begin(), pos_first.end(), s) - pos_first.begin()) - 1;
                for(uint64_t a = s; a < e; ++i)
                {
                    const uint64_t b = std::min<uint64_t>(e, pos_first[i + 1]), m = b - a, at = a - pos_first[i];
                    if(m == 0)
                        continue;
                    std::memcpy(static_cast<uint8_t*>(g[i]->out0) + at, f + a, m);
                    if(g[i]->out1 && vb)
                        std::memcpy(static_cast<uint8_t*>(g[i]->out1) + at * vb, vals + a * vb, m * vb);
                    if(g[i]->out2)
                        std::memcpy(static_cast<uint8_t*>(g[i]->out2) + at, fw + a, m);
                    uint64_t c = 0;
                    for(uint64_t j = a; j < b; ++j)
                        c += f[j] == 1;
                    hits[i] += c;
                    a = b;
                }
            });
            for(size_t i = 0; i < g.size(); ++i)
                g[i]->result = hits[i].load();
        }
        else
        {
            counts.ensure((n + 1) * 8);
            const uint64_t* c = counts.as<uint64_t>();
            t->seq_reduce(seqs.data(), lens.data(), n, 0, 0, 0, counts.as<uint64_t>());
            for(size_t i = 0; i < g.size(); ++i)
            {
                uint64_t s = 0;
                for(size_t q = first[i]; q < first[i + 1]; ++q)
                    s += c[q];
                std::memcpy(g[i]->out0, c + first[i], (first[i + 1] - first[i]) * sizeof(uint64_t));
                g[i]->result = s;
            }
        }
    }
    catch(const std::bad_alloc&)
    {
        for(Request* r : g)
            r->status = KACHE_ENOMEM;
    }
    catch(...)
    {
        for(Request* r : g)
            r->status = KACHE_EINTERNAL;
    }
}

extern "C" int kache_b200_server_new(kache_table* const t, const uint64_t budget_bytes, kache_server** const out) noexcept
{
    if(t == nullptr || out == nullptr)
        return KACHE_EINVAL;
    *out = nullptr;
    try
    {
        uint32_t user = 0;
        {
            std::lock_guard<std::mutex> g(t->reg);
            if(t->user_c.load() >= KACHE_MAX_USERS)
                return KACHE_EUSERS;
            user = t->user_c++;
        }
        auto* s = new kache_server;
        s->t = t, s->user = user;
        size_t free_b = 0, total_b = 0;
        if(cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
            free_b = size_t(1) << 30;
        // The budget: as asked, but at most half the device memory free now.
        s->budget = std::max<uint64_t>(1, std::min<uint64_t>(budget_bytes ? budget_bytes : ~0ull, free_b / 2));
        // The merged outputs of a full-size run, page-locked once here rather than while requests wait.
        const uint64_t P = kache_server::run_positions;
        s->found.ensure(P + 16), s->values.ensure(P * std::max<uint32_t>(1, t->value_bytes) + 16);
        s->counts.ensure((P / 16) * 8);
        // Staging for the bases of a full-size run of reads of 100 bp or more (positions x 1.5), in both buffers.
        s->stage[0].ensure(P * 3 / 2), s->stage[1].ensure(P * 3 / 2);
        s->executor = std::thread([s](){ s->execute(); });
        s->worker = std::thread([s](){ s->loop(); });
        *out = s;
        return KACHE_OK;
    }
    catch(const std::bad_alloc&)
    {
        return KACHE_ENOMEM;
    }
    catch(...)
    {
        return KACHE_EINTERNAL;
    }
}

extern "C" void kache_b200_server_free(kache_server* const s) noexcept
{
    if(s == nullptr)
        return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if(s->worker.joinable())
        s->worker.join();
    if(s->executor.joinable())
        s->executor.join();
    for(auto& kv : s->all)
        delete kv.second;
    delete s;
}

extern "C" int kache_b200_server_submit(kache_server* const s, const uint32_t kind, const char* const* const seqs, const size_t* const lens, const size_t n,
                                        const uint32_t op, const uint64_t x, const uint64_t init, void* const out0, void* const out1, void* const out2,
                                        uint64_t* const ticket) noexcept
{
    if(s == nullptr || ticket == nullptr || kind > KACHE_B200_REQ_COUNT || (n > 0 && (seqs == nullptr || lens == nullptr)))
        return KACHE_EINVAL;
    if(kind != KACHE_B200_REQ_UPSERT && n > 0 && out0 == nullptr)
        return KACHE_EINVAL;
    if(kind == KACHE_B200_REQ_UPSERT && op != KACHE_B200_ADD_WRAP && op > KACHE_MAX)
        return KACHE_EINVAL;
    try
    {
        auto* r = new Request;
        r->kind = kind, r->op = op, r->x = x, r->init = init, r->out0 = out0, r->out1 = out1, r->out2 = out2;
        r->seqs.assign(seqs, seqs + n), r->lens.assign(lens, lens + n);
        const uint32_t k = s->t->kmer_k;
        for(const size_t len : r->lens)
            r->positions += len >= k ? len - k + 1 : 0;
        r->bytes = request_bytes(*r, k, s->t->value_bytes);
        r->t_submit = clock_type::now();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->ticket = s->next_ticket++;
            s->all[r->ticket] = r;
            s->queue.push_back(r);
        }
        s->cv.notify_one();
        *ticket = r->ticket;
        return KACHE_OK;
    }
    catch(const std::bad_alloc&)
    {
        return KACHE_ENOMEM;
    }
}

extern "C" int kache_b200_server_submit_dev(kache_server* const s, const uint32_t kind, const uint8_t* const d_bases, const uint64_t* const d_off,
                                            const uint64_t n, const uint32_t op, const uint64_t x, const uint64_t init, void* const out0,
                                            void* const out1, void* const out2, uint64_t* const ticket) noexcept
{
    if(s == nullptr || ticket == nullptr || kind > KACHE_B200_REQ_COUNT || (n > 0 && (d_bases == nullptr || d_off == nullptr)))
        return KACHE_EINVAL;
    if(kind != KACHE_B200_REQ_UPSERT && n > 0 && out0 == nullptr)
        return KACHE_EINVAL;
    if(kind == KACHE_B200_REQ_UPSERT && op != KACHE_B200_ADD_WRAP && op > KACHE_MAX)
        return KACHE_EINVAL;
    if(kind == KACHE_B200_REQ_LOOKUP && s->t->value_bytes == 0 && out1 != nullptr)
        return KACHE_EINVAL;
    try
    {
        auto* r = new Request;
        r->kind = kind, r->op = op, r->x = x, r->init = init, r->out0 = out0, r->out1 = out1, r->out2 = out2;
        r->dev = true, r->d_bases = d_bases, r->d_off = d_off, r->n_dev = n;
        // Nothing is read from the device here: a submission never waits for the GPU. Device bytes of its share of
        // the merged list: offsets, addresses, lengths, per-sequence results and batch numbers, 36 bytes a sequence.
        r->bytes = 36 * n + 64;
        r->t_submit = clock_type::now();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->ticket = s->next_ticket++;
            s->all[r->ticket] = r;
            s->queue.push_back(r);
        }
        s->cv.notify_one();
        *ticket = r->ticket;
        return KACHE_OK;
    }
    catch(const std::bad_alloc&)
    {
        return KACHE_ENOMEM;
    }
}

extern "C" int kache_b200_server_wait(kache_server* const s, const uint64_t ticket, uint64_t* const result, double* const latency_ms) noexcept
{
    if(s == nullptr)
        return KACHE_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    const auto it = s->all.find(ticket);
    if(it == s->all.end())
        return KACHE_EINVAL;
    Request* r = it->second;
    s->done_cv.wait(lk, [&](){ return r->done; });
    if(result)
        *result = r->result;
    if(latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    const int status = r->status;
    s->all.erase(it);
    delete r;
    return status;
}

extern "C" int kache_b200_server_stats(kache_server* const s, uint64_t* const runs, uint64_t* const requests) noexcept
{
    if(s == nullptr)
        return KACHE_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if(runs)
        *runs = s->runs;
    if(requests)
        *requests = s->merged;
    return KACHE_OK;
}
