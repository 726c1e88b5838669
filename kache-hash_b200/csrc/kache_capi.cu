// The C interface (include/kache_capi.h, include/kache_b200.h) over the B200 engine.
//
// Argument validation, status codes and the user bound follow the reference's capi/kache_capi.cpp:15-289 so that
// the two libraries answer every call alike: validation before any work, every exception caught (std::bad_alloc as
// KACHE_ENOMEM, anything else, a CUDA failure included, as KACHE_EINTERNAL).
#include "engine.cuh"
#include "kache_b200.h"
#include "kache_b200_testing.h"

#include <exception>
#include <mutex>
#include <new>

namespace kache_b200
{

std::atomic<uint64_t>& launches()
{
    static std::atomic<uint64_t> n{0};
    return n;
}

std::atomic<int64_t>& alloc_fail_countdown()
{
    static std::atomic<int64_t> c{-1};
    return c;
}

// The engine's instantiations, one translation unit per (k, l) (tables_<k>_<l>.cu).
kache_table* make_table_31_22(uint32_t vb, uint64_t n, double lf, bool pow2);
kache_table* make_table_27_16(uint32_t vb, uint64_t n, double lf, bool pow2);
kache_table* make_table_32_20(uint32_t vb, uint64_t n, double lf, bool pow2);

kache_table* make_table(const uint32_t k, const uint32_t l, const uint32_t vb, const uint64_t n, const double lf, const bool pow2)
{
    if(k == 31 && l == 22)
        return make_table_31_22(vb, n, lf, pow2);
    if(k == 27 && l == 16)
        return make_table_27_16(vb, n, lf, pow2);
    if(k == 32 && l == 20)
        return make_table_32_20(vb, n, lf, pow2);
    return nullptr;
}

bool supported_kl(const uint32_t k, const uint32_t l) { return (k == 31 && l == 22) || (k == 27 && l == 16) || (k == 32 && l == 20); }
bool supported_vb(const uint32_t vb) { return vb == 0 || vb == 1 || vb == 2 || vb == 4 || vb == 8; }

}

namespace
{

using namespace kache_b200;

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
    catch(...)
    {
        return KACHE_EINTERNAL;
    }
}

// Only empty sequences may be NULL (capi/kache_capi.cpp:32-46).
bool valid(const char* const* seqs, const size_t* lens, const size_t n)
{
    if(n == 0)
        return true;
    if(seqs == nullptr || lens == nullptr)
        return false;
    for(size_t i = 0; i < n; ++i)
        if(seqs[i] == nullptr && lens[i] > 0)
            return false;
    return true;
}

// A map whose values the operand fits (capi/kache_capi.cpp:49-53).
bool fits_x(const kache_table* t, const uint64_t x) { return t->value_bytes > 0 && (t->value_bytes == 8 || x >> (8 * t->value_bytes) == 0); }

bool registered(const kache_table* t, const uint32_t user) { return user < t->user_c.load(std::memory_order_acquire); }

bool oriented_op_ok(const uint32_t op, const bool wrap) { return op == KACHE_ASSIGN || op == KACHE_ADD || op == KACHE_OR || op == KACHE_MAX || (wrap && op == KACHE_B200_ADD_WRAP); }

int new_table(const uint32_t k, const uint32_t l, const uint32_t vb, const uint64_t n, const double lf, const uint32_t pow2, kache_table** out)
{
    if(out == nullptr)
        return KACHE_EINVAL;
    *out = nullptr;
    if(!supported_kl(k, l) || !supported_vb(vb) || !(lf > 0 && lf < 1) || pow2 > 1 || !kache_b200::fits(n, lf, pow2 != 0))
        return KACHE_EINVAL;
    return guard([&]()
    {
        *out = make_table(k, l, vb, n, lf, pow2 != 0);
        return *out ? KACHE_OK : KACHE_EINVAL;
    });
}

}

extern "C"
{

int kache_supports(const uint32_t k, const uint32_t value_bytes) noexcept
{
    return k == 31 && supported_vb(value_bytes);
}

kache_options kache_default_options(const uint32_t k, const uint32_t value_bytes) noexcept
{
    return kache_options{k, value_bytes, uint64_t(1) << 22, 0.8, 16, 0};
}

int kache_new(const kache_options* const options, kache_table** const out) noexcept
{
    if(out == nullptr)
        return KACHE_EINVAL;
    *out = nullptr;
    if(options == nullptr)
        return KACHE_EINVAL;
    const auto& o = *options;
    if(!kache_supports(o.k, o.value_bytes) || o.resize_workers < 1)
        return KACHE_EINVAL;
    return new_table(o.k, 22, o.value_bytes, o.expected_keys, o.load_factor, o.pow2_capacity, out);
}

void kache_free(kache_table* const t) noexcept
{
    delete t;
}

int kache_register(kache_table* const t, uint32_t* const user) noexcept
{
    if(t == nullptr || user == nullptr)
        return KACHE_EINVAL;
    return guard([&]()
    {
        const std::lock_guard<std::mutex> lock(t->reg);
        const auto u = t->user_c.load(std::memory_order_relaxed);
        if(u == KACHE_MAX_USERS)
            return KACHE_EUSERS;
        t->user_c.store(u + 1, std::memory_order_release);
        *user = u;
        return KACHE_OK;
    });
}

int kache_insert(kache_table* const t, const uint32_t user, const char* const* const seqs, const size_t* const lens, const size_t n, const uint32_t op, const uint64_t x, uint64_t* const inserted) noexcept
{
    if(t == nullptr || !registered(t, user) || !valid(seqs, lens, n) || (t->value_bytes > 0 && (op > KACHE_MAX || !fits_x(t, x))))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->upsert(user, seqs, lens, n, op, x, x);
        if(inserted != nullptr)
            *inserted = c;
        return KACHE_OK;
    });
}

int kache_insert_oriented(kache_table* const t, const uint32_t user, const char* const* const seqs, const size_t* const lens, const size_t n, const uint32_t op, const uint64_t x_fwd, const uint64_t x_rev, uint64_t* const inserted) noexcept
{
    if(t == nullptr || !registered(t, user) || !valid(seqs, lens, n) || !oriented_op_ok(op, false) || !fits_x(t, x_fwd) || !fits_x(t, x_rev))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->upsert_oriented(user, seqs, lens, n, op, x_fwd, x_rev);
        if(inserted != nullptr)
            *inserted = c;
        return KACHE_OK;
    });
}

int kache_update(kache_table* const t, const char* const* const seqs, const size_t* const lens, const size_t n, const uint32_t op, const uint64_t x, uint64_t* const present) noexcept
{
    if(t == nullptr || !valid(seqs, lens, n) || op > KACHE_MAX || !fits_x(t, x))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->update(seqs, lens, n, op, x);
        if(present != nullptr)
            *present = c;
        return KACHE_OK;
    });
}

int kache_count(const kache_table* const t, const char* const* const seqs, const size_t* const lens, const size_t n, uint64_t* const counts) noexcept
{
    if(t == nullptr || !valid(seqs, lens, n) || (n > 0 && counts == nullptr))
        return KACHE_EINVAL;
    return guard([&](){ return const_cast<kache_table*>(t)->seq_reduce(seqs, lens, n, 0, 0, 0, counts), KACHE_OK; });
}

int kache_count_masked(const kache_table* const t, const char* const* const seqs, const size_t* const lens, const size_t n, const uint64_t mask_fwd, const uint64_t mask_rev, uint64_t* const counts) noexcept
{
    if(t == nullptr || t->value_bytes == 0 || !valid(seqs, lens, n) || (n > 0 && counts == nullptr))
        return KACHE_EINVAL;
    return guard([&](){ return const_cast<kache_table*>(t)->seq_reduce(seqs, lens, n, 1, mask_fwd, mask_rev, counts), KACHE_OK; });
}

int kache_sum(const kache_table* const t, const char* const* const seqs, const size_t* const lens, const size_t n, uint64_t* const sums) noexcept
{
    if(t == nullptr || t->value_bytes == 0 || !valid(seqs, lens, n) || (n > 0 && sums == nullptr))
        return KACHE_EINVAL;
    return guard([&](){ return const_cast<kache_table*>(t)->seq_reduce(seqs, lens, n, 2, 0, 0, sums), KACHE_OK; });
}

int kache_lookup(const kache_table* const t, const char* const* const seqs, const size_t* const lens, const size_t n, uint8_t* const found, void* const values, uint8_t* const fwd) noexcept
{
    if(t == nullptr || !valid(seqs, lens, n) || (n > 0 && found == nullptr) || (t->value_bytes == 0 && values != nullptr))
        return KACHE_EINVAL;
    return guard([&](){ return const_cast<kache_table*>(t)->lookup(seqs, lens, n, found, values, fwd), KACHE_OK; });
}

int kache_get(const kache_table* const t, const char* const kmer, uint8_t* const found, uint64_t* const value) noexcept
{
    if(t == nullptr || kmer == nullptr || found == nullptr)
        return KACHE_EINVAL;
    return guard([&]()
    {
        uint64_t v = 0;
        *found = const_cast<kache_table*>(t)->get(kmer, v);
        if(value != nullptr)
            *value = v;
        return KACHE_OK;
    });
}

int kache_size(const kache_table* const t, uint64_t* const keys) noexcept
{
    if(t == nullptr || keys == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return *keys = t->size(), KACHE_OK; });
}

int kache_reduce(const kache_table* const t, const uint32_t what, const uint64_t mask, const uint32_t workers, uint64_t* const out) noexcept
{
    if(t == nullptr || out == nullptr || workers < 1 || what > KACHE_REDUCE_SUM || (t->value_bytes == 0 && what != KACHE_REDUCE_KEYS))
        return KACHE_EINVAL;
    return guard([&](){ return *out = const_cast<kache_table*>(t)->reduce(what, mask), KACHE_OK; });
}

int kache_for_each(const kache_table* const t, const uint32_t shards, const uint32_t shard, const kache_keys_fn f, void* const ctx) noexcept
{
    if(t == nullptr || f == nullptr || shard >= shards)
        return KACHE_EINVAL;
    return guard([&](){ return const_cast<kache_table*>(t)->for_each(shards, shard, f, ctx), KACHE_OK; });
}

int kache_get_stats(const kache_table* const t, kache_stats* const out) noexcept
{
    if(t == nullptr || out == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return const_cast<kache_table*>(t)->get_stats(*out), KACHE_OK; });
}

const char* kache_strerror(const int code) noexcept
{
    switch(code)
    {
    case KACHE_OK: return "success";
    case KACHE_EINVAL: return "invalid argument";
    case KACHE_EUSERS: return "too many users registered";
    case KACHE_ENOMEM: return "out of memory";
    case KACHE_EINTERNAL: return "internal error";
    default: return "unknown status";
    }
}

// ---- Extensions ----

int kache_b200_new(const uint32_t k, const uint32_t l, const uint32_t value_bytes, const uint64_t expected_keys, const double load_factor, const uint32_t pow2_capacity, kache_table** const out) noexcept
{
    return new_table(k, l, value_bytes, expected_keys, load_factor, pow2_capacity, out);
}

int kache_b200_set_stream(kache_table* const t, void* const stream) noexcept
{
    if(t == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return t->set_stream(static_cast<cudaStream_t>(stream)), KACHE_OK; });
}

static bool op_ok(const uint32_t op) { return op <= KACHE_MAX || op == KACHE_B200_ADD_WRAP; }

int kache_b200_upsert(kache_table* const t, const uint32_t user, const char* const* const seqs, const size_t* const lens, const size_t n, const uint32_t op, const uint64_t x, const uint64_t init, uint64_t* const inserted) noexcept
{
    if(t == nullptr || !registered(t, user) || !valid(seqs, lens, n) || (t->value_bytes > 0 && !op_ok(op)))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->upsert(user, seqs, lens, n, op, x, init);
        if(inserted != nullptr)
            *inserted = c;
        return KACHE_OK;
    });
}

int kache_b200_upsert_oriented(kache_table* const t, const uint32_t user, const char* const* const seqs, const size_t* const lens, const size_t n, const uint32_t op, const uint64_t x_fwd, const uint64_t x_rev, uint64_t* const inserted) noexcept
{
    if(t == nullptr || t->value_bytes == 0 || !registered(t, user) || !valid(seqs, lens, n) || !oriented_op_ok(op, true))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->upsert_oriented(user, seqs, lens, n, op, x_fwd, x_rev);
        if(inserted != nullptr)
            *inserted = c;
        return KACHE_OK;
    });
}

int kache_b200_update(kache_table* const t, const char* const* const seqs, const size_t* const lens, const size_t n, const uint32_t op, const uint64_t x, uint64_t* const present) noexcept
{
    if(t == nullptr || t->value_bytes == 0 || !valid(seqs, lens, n) || !op_ok(op))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->update(seqs, lens, n, op, x);
        if(present != nullptr)
            *present = c;
        return KACHE_OK;
    });
}

int kache_b200_upsert_dev(kache_table* const t, const uint32_t user, const uint8_t* const d_bases, const uint64_t* const d_off, const uint64_t n, const uint32_t op, const uint64_t x, const uint64_t init, uint64_t* const inserted) noexcept
{
    if(t == nullptr || !registered(t, user) || (n > 0 && (d_bases == nullptr || d_off == nullptr)) || (t->value_bytes > 0 && !op_ok(op)))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->upsert_dev(user, d_bases, d_off, n, op, x, init);
        if(inserted != nullptr)
            *inserted = c;
        return KACHE_OK;
    });
}

int kache_b200_upsert_oriented_dev(kache_table* const t, const uint32_t user, const uint8_t* const d_bases, const uint64_t* const d_off, const uint64_t n, const uint32_t op, const uint64_t x_fwd, const uint64_t x_rev, uint64_t* const inserted) noexcept
{
    if(t == nullptr || t->value_bytes == 0 || !registered(t, user) || (n > 0 && (d_bases == nullptr || d_off == nullptr)) || !oriented_op_ok(op, true))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->upsert_oriented_dev(user, d_bases, d_off, n, op, x_fwd, x_rev);
        if(inserted != nullptr)
            *inserted = c;
        return KACHE_OK;
    });
}

int kache_b200_update_dev(kache_table* const t, const uint8_t* const d_bases, const uint64_t* const d_off, const uint64_t n, const uint32_t op, const uint64_t x, uint64_t* const present) noexcept
{
    if(t == nullptr || t->value_bytes == 0 || (n > 0 && (d_bases == nullptr || d_off == nullptr)) || !op_ok(op))
        return KACHE_EINVAL;
    return guard([&]()
    {
        const auto c = t->update_dev(d_bases, d_off, n, op, x);
        if(present != nullptr)
            *present = c;
        return KACHE_OK;
    });
}

int kache_b200_lookup_dev(kache_table* const t, const uint8_t* const d_bases, const uint64_t* const d_off, const uint64_t n, uint8_t* const d_found, void* const d_values, uint8_t* const d_fwd) noexcept
{
    if(t == nullptr || (n > 0 && (d_bases == nullptr || d_off == nullptr || d_found == nullptr)) || (t->value_bytes == 0 && d_values != nullptr))
        return KACHE_EINVAL;
    return guard([&](){ return t->lookup_dev(d_bases, d_off, n, d_found, d_values, d_fwd), KACHE_OK; });
}

int kache_b200_count_dev(kache_table* const t, const uint8_t* const d_bases, const uint64_t* const d_off, const uint64_t n, uint64_t* const d_counts) noexcept
{
    if(t == nullptr || (n > 0 && (d_bases == nullptr || d_off == nullptr || d_counts == nullptr)))
        return KACHE_EINVAL;
    return guard([&](){ return t->count_dev(d_bases, d_off, n, d_counts), KACHE_OK; });
}

int kache_b200_run_dev_batches(kache_table* const t, const uint32_t user, const uint32_t kind, const uint32_t op, const uint64_t x, const uint64_t y, kache_dev_batch* const batches, const size_t count) noexcept
{
    if(t == nullptr || kind > KACHE_B200_RUN_COUNT || (count > 0 && batches == nullptr) || count > (size_t(1) << 32))
        return KACHE_EINVAL;
    const bool upsert = kind == KACHE_B200_RUN_UPSERT || kind == KACHE_B200_RUN_UPSERT_ORIENTED;
    if(upsert && !registered(t, user))
        return KACHE_EINVAL;
    if(kind == KACHE_B200_RUN_UPSERT && t->value_bytes > 0 && !op_ok(op))
        return KACHE_EINVAL;
    if(kind == KACHE_B200_RUN_UPSERT_ORIENTED && (t->value_bytes == 0 || !oriented_op_ok(op, true)))
        return KACHE_EINVAL;
    if(kind == KACHE_B200_RUN_UPDATE && (t->value_bytes == 0 || !op_ok(op)))
        return KACHE_EINVAL;
    for(size_t b = 0; b < count; ++b)
    {
        const kache_dev_batch& e = batches[b];
        if(e.n > 0 && (e.d_bases == nullptr || e.d_off == nullptr))
            return KACHE_EINVAL;
        if(e.n > 0 && (kind == KACHE_B200_RUN_LOOKUP || kind == KACHE_B200_RUN_COUNT) && e.out0 == nullptr)
            return KACHE_EINVAL;
        if(kind == KACHE_B200_RUN_LOOKUP && t->value_bytes == 0 && e.out1 != nullptr)
            return KACHE_EINVAL;
    }
    return guard([&](){ return t->run_dev_batches(user, kind, op, x, y, batches, count), KACHE_OK; });
}

int kache_b200_prepare_dev(kache_table* const t, const uint64_t* const d_off, const uint64_t n, kache_prepared** const out) noexcept
{
    if(t == nullptr || out == nullptr || (n > 0 && d_off == nullptr))
        return KACHE_EINVAL;
    *out = nullptr;
    return guard([&](){ return *out = t->prepare_dev(d_off, n), KACHE_OK; });
}

void kache_b200_prepared_free(kache_prepared* const p) noexcept
{
    delete p;
}

int kache_b200_lookup_prepared(kache_table* const t, const kache_prepared* const p, const uint8_t* const d_bases, uint8_t* const d_found,
                               void* const d_values, uint8_t* const d_fwd) noexcept
{
    if(t == nullptr || p == nullptr || p->t != t)
        return KACHE_EINVAL;
    if(p->total_pos > 0 && (d_bases == nullptr || d_found == nullptr))
        return KACHE_EINVAL;
    if(t->value_bytes == 0 && d_values != nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return t->lookup_prepared(*p, d_bases, d_found, d_values, d_fwd), KACHE_OK; });
}

int kache_b200_count_prepared(kache_table* const t, const kache_prepared* const p, const uint8_t* const d_bases, uint64_t* const d_counts) noexcept
{
    if(t == nullptr || p == nullptr || p->t != t)
        return KACHE_EINVAL;
    if(p->n > 0 && (d_bases == nullptr || d_counts == nullptr))
        return KACHE_EINVAL;
    return guard([&](){ return t->count_prepared(*p, d_bases, d_counts), KACHE_OK; });
}

int kache_b200_table_epoch(kache_table* const t, uint64_t* const epoch) noexcept
{
    if(t == nullptr || epoch == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return *epoch = t->epoch(), KACHE_OK; });
}

int kache_b200_describe(kache_table* const t, const char* const* const seqs, const size_t* const lens, const size_t n, uint64_t* const key, uint64_t* const h, uint8_t* const cs, uint8_t* const fwd, uint8_t* const valid_out) noexcept
{
    if(t == nullptr || !valid(seqs, lens, n) || !key || !h || !cs || !fwd || !valid_out)
        return KACHE_EINVAL;
    return guard([&](){ return t->describe(seqs, lens, n, key, h, cs, fwd, valid_out), KACHE_OK; });
}

int kache_b200_histogram(kache_table* const t, const uint64_t max, uint64_t* const h) noexcept
{
    if(t == nullptr || h == nullptr || t->value_bytes == 0)
        return KACHE_EINVAL;
    return guard([&](){ return t->histogram(max, h), KACHE_OK; });
}

int kache_b200_clear(kache_table* const t) noexcept
{
    if(t == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return t->clear(), KACHE_OK; });
}

int kache_b200_profile(kache_table* const t, const int on) noexcept
{
    if(t == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return t->profile(on != 0), KACHE_OK; });
}

int kache_b200_profile_read(kache_table* const t, const uint32_t kind, double* const ms, uint64_t* const n) noexcept
{
    if(t == nullptr || ms == nullptr || n == nullptr)
        return KACHE_EINVAL;
    return guard([&](){ return t->profile_read(kind, *ms, *n), KACHE_OK; });
}

uint64_t kache_b200_kernel_launches(void) noexcept
{
    return kache_b200::launches().load();
}

int kache_b200_testing_fail_allocation(const int64_t after) noexcept
{
    kache_b200::alloc_fail_countdown().store(after < 0 ? -1 : after);
    return KACHE_OK;
}

int kache_b200_testing_plant_claim(kache_table* const t, const char* const kmer, const uint32_t wait_polls) noexcept
{
    if(t == nullptr || kmer == nullptr)
        return KACHE_EINVAL;
    uint64_t f = 0, r = 0;
    for(uint32_t i = 0; i < t->kmer_k; ++i)
    {
        const char c = static_cast<char>(kmer[i] | 0x20);
        if(c != 'a' && c != 'c' && c != 'g' && c != 't')
            return KACHE_EINVAL;
        const uint64_t b = static_cast<uint64_t>(((kmer[i] >> 2) ^ (kmer[i] >> 1)) & 3);
        f = (f << 2) | b;
        r |= (3 - b) << (2 * i);
    }
    const uint64_t key = f < r ? f : r;
    return guard([&]()
    {
        uint64_t v = 0;
        if(t->get(kmer, v))
            return KACHE_EINVAL;
        t->testing_wait_polls(wait_polls);
        return t->testing_plant_claim(key) ? KACHE_OK : KACHE_EINVAL;
    });
}

}
