/* CPU restatement of kache-hash's streaming k-mer table semantics; see oracle.h for what it restates and where.
 * TEST INFRASTRUCTURE ONLY: the checker, never the product. */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Thomas Wang's 64-bit hash, as Kmer_Batch.hpp:24-35 defines it. */
uint64_t orc_wang(uint64_t x)
{
    x = (~x) + (x << 21);
    x = x ^ (x >> 24);
    x = (x + (x << 3)) + (x << 8);
    x = x ^ (x >> 14);
    x = (x + (x << 2)) + (x << 4);
    x = x ^ (x >> 28);
    x = x + (x << 31);
    return x;
}

/* The checksum of a canonical key: the top byte of key * 0x9E3779B97F4A7C15, 0 mapped to 1
 * (Kmer_Batch.hpp:44-67, the variant built without AVX-512). */
uint8_t orc_checksum(const uint64_t key)
{
    const uint8_t c = (uint8_t)((key * 0x9E3779B97F4A7C15ull) >> 56);
    return c ? c : 1;
}

static uint64_t mask_of(const int k) { return k == 32 ? ~0ull : (1ull << (2 * k)) - 1; }

uint64_t orc_revcomp(const uint64_t x, const int k)
{
    uint64_t r = 0, y = x;
    for(int i = 0; i < k; ++i, y >>= 2)
        r = (r << 2) | (3 - (y & 3));
    return r;
}

/* The least Wang hash of the canonical forms of the key's l-mers (Kmer_Lanes.hpp:247-274): a k-mer and its reverse
 * complement share it. */
uint64_t orc_minimizer_hash(const uint64_t key, const int k, const int l)
{
    const uint64_t lm = mask_of(l);
    uint64_t h = ~0ull;
    for(int p = 0; p + l <= k; ++p)
    {
        const uint64_t f = (key >> (2 * (k - l - p))) & lm;
        const uint64_t r = orc_revcomp(f, l);
        const uint64_t x = orc_wang(f < r ? f : r);
        if(x < h)
            h = x;
    }
    return h;
}

static int is_acgt(const char c)
{
    const char x = (char)(c | 0x20);
    return x == 'a' || x == 'c' || x == 'g' || x == 't';
}

static uint64_t code(const char c) { return (uint64_t)(((c >> 2) ^ (c >> 1)) & 3); }

uint64_t orc_describe(const char* s, const uint64_t len, const int k, const int l, uint64_t* key, uint64_t* h, uint8_t* cs, uint8_t* fwd, uint8_t* valid)
{
    if(len < (uint64_t)k)
        return 0;
    const uint64_t n = len - k + 1, km = mask_of(k);
    uint64_t f = 0, r = 0, run = 0;
    for(uint64_t j = 0; j < len; ++j)
    {
        if(!is_acgt(s[j]))
            run = 0;
        else
        {
            const uint64_t b = code(s[j]);
            f = ((f << 2) | b) & km;
            r = (r >> 2) | ((3 - b) << (2 * (k - 1)));
            run++;
        }
        if(j + 1 < (uint64_t)k)
            continue;
        const uint64_t i = j + 1 - k;
        if(run >= (uint64_t)k)
        {
            /* Canonical = the lesser form; a palindrome counts as forward (Kmer_Batch.hpp:236-240). */
            const uint64_t c = f < r ? f : r;
            key[i] = c, h[i] = orc_minimizer_hash(c, k, l), cs[i] = orc_checksum(c), fwd[i] = (c == f), valid[i] = 1;
        }
        else
            key[i] = 0, h[i] = 0, cs[i] = 0, fwd[i] = 0, valid[i] = 0;
    }
    return n;
}

static uint64_t ceil_pow2(uint64_t x)
{
    uint64_t p = 1;
    while(p < x)
        p <<= 1;
    return p;
}

enum { B = 32 };
static const uint64_t max_cap = (1ull << 32) - 1;
static const uint64_t max_user = 128;

/* Streaming_Kmer_Hash_Table.hpp:1004-1011. */
uint64_t orc_cap_for(const uint64_t max_sz, const double lf, const int pow2)
{
    uint64_t cap = (uint64_t)ceil((double)max_sz / lf / B);
    if(cap < 1)
        cap = 1;
    while((uint64_t)((double)(cap * B) * lf) <= max_sz)
        cap++;
    return pow2 ? ceil_pow2(cap) : cap;
}

/* Streaming_Kmer_Hash_Table.hpp:800-804. */
int orc_fits(const uint64_t max_sz, const double lf, const int pow2)
{
    return (double)max_sz / lf / B <= (double)max_cap && orc_cap_for(max_sz, lf, pow2) <= max_cap;
}

/* Streaming_Kmer_Hash_Table.hpp:383. */
static uint64_t step_for(const uint64_t th)
{
    uint64_t s = th / (8 * max_user);
    return s < 1 ? 1 : (s > 16384 ? 16384 : s);
}

/* The exact dictionary: open addressing over keys, all-ones marking empty slots (no canonical k-mer is all T's). */
struct orc_table
{
    int k, vb;
    double lf;
    uint64_t vmask;
    uint64_t* key;
    uint64_t* val;
    uint64_t slots, n;
    /* The resize schedule's state (Streaming_Kmer_Hash_Table.hpp:224-229). */
    uint64_t cap, resize_th, step, approx_sz;
    uint64_t pending[128];
    uint32_t users;
};

static const uint64_t EMPTY = ~0ull;

static uint64_t mix(uint64_t x)
{
    x ^= x >> 33, x *= 0xff51afd7ed558ccdull, x ^= x >> 33, x *= 0xc4ceb9fe1a85ec53ull, x ^= x >> 33;
    return x;
}

static uint64_t* slot_of(const orc_table* t, const uint64_t k)
{
    uint64_t i = mix(k) & (t->slots - 1);
    while(t->key[i] != EMPTY && t->key[i] != k)
        i = (i + 1) & (t->slots - 1);
    return &t->key[i];
}

static void grow(orc_table* t)
{
    uint64_t* ok = t->key;
    uint64_t* ov = t->val;
    const uint64_t os = t->slots;
    t->slots = os * 2;
    t->key = malloc(t->slots * sizeof(uint64_t));
    t->val = malloc(t->slots * sizeof(uint64_t));
    memset(t->key, 0xFF, t->slots * sizeof(uint64_t));
    for(uint64_t i = 0; i < os; ++i)
        if(ok[i] != EMPTY)
        {
            uint64_t* p = slot_of(t, ok[i]);
            *p = ok[i], t->val[p - t->key] = ov[i];
        }
    free(ok), free(ov);
}

orc_table* orc_new(const int k, const int value_bytes, const uint64_t max_sz, const double lf, const int pow2)
{
    orc_table* t = calloc(1, sizeof(orc_table));
    t->k = k, t->vb = value_bytes, t->lf = lf;
    t->vmask = value_bytes == 8 ? ~0ull : (value_bytes == 0 ? 0 : (1ull << (8 * value_bytes)) - 1);
    t->slots = 1024;
    t->key = malloc(t->slots * sizeof(uint64_t));
    t->val = malloc(t->slots * sizeof(uint64_t));
    memset(t->key, 0xFF, t->slots * sizeof(uint64_t));
    t->cap = orc_cap_for(max_sz, lf, pow2);
    t->resize_th = (uint64_t)((double)(t->cap * B) * lf);
    t->step = step_for(t->resize_th);
    return t;
}

void orc_free(orc_table* t)
{
    if(!t)
        return;
    free(t->key), free(t->val), free(t);
}

uint32_t orc_register(orc_table* t) { return t->users++; }

/* The C interface's operations (capi/Kmer_Table.hpp:30-43), and the wrapping add of the template API's `v + x`. */
static uint64_t apply(const orc_table* t, const uint32_t op, const uint64_t v, uint64_t x)
{
    const uint64_t mx = t->vmask;
    x &= mx;
    switch(op)
    {
    case ORC_KEEP: return v;
    case ORC_ASSIGN: return x;
    case ORC_ADD: return v > mx - x ? mx : v + x;
    case ORC_OR: return v | x;
    case ORC_MIN: return v < x ? v : x;
    case ORC_ADD_WRAP: return (v + x) & mx;
    default: return v > x ? v : x;
    }
}

/* Accounts for `ins` keys newly inserted by `user` in one call, doubling the capacity where the reference would:
 * every `step` keys a user flushes its count into the table's, and a flush that reaches the threshold resizes
 * (Streaming_Kmer_Hash_Table.hpp:2244-2286, 1447-1455, 1679-1680). */
static void account(orc_table* t, const uint32_t user, const uint64_t ins)
{
    uint64_t pending = t->pending[user], flushed = 0;
    uint64_t due = pending < t->step ? t->step - pending : 1;
    while(due <= ins)
    {
        const uint64_t at = due;
        t->approx_sz += pending + (at - flushed);
        pending = 0, flushed = at, due = at + t->step;
        if(t->approx_sz >= t->resize_th)
        {
            t->cap *= 2;
            t->resize_th = (uint64_t)((double)(t->cap * B) * t->lf);
            t->step = step_for(t->resize_th);
        }
    }
    t->pending[user] = pending + (ins - flushed);
}

/* Calls f(ctx, q, i, key, fwd) on each k-mer of each sequence, in order. */
typedef void (*visit_fn)(void* ctx, uint64_t q, uint64_t i, uint64_t key, int fwd);

static void stream(const int k, const char* bases, const uint64_t* off, const uint64_t n, visit_fn f, void* ctx)
{
    const uint64_t km = mask_of(k);
    for(uint64_t q = 0; q < n; ++q)
    {
        const char* s = bases + off[q];
        const uint64_t len = off[q + 1] - off[q];
        uint64_t fw = 0, rv = 0, run = 0;
        for(uint64_t j = 0; j < len; ++j)
        {
            if(!is_acgt(s[j]))
            {
                run = 0;
                continue;
            }
            const uint64_t b = code(s[j]);
            fw = ((fw << 2) | b) & km;
            rv = (rv >> 2) | ((3 - b) << (2 * (k - 1)));
            if(++run >= (uint64_t)k)
                f(ctx, q, j + 1 - k, fw < rv ? fw : rv, fw <= rv);
        }
    }
}

struct up_ctx
{
    orc_table* t;
    uint32_t op;
    uint64_t x, init, x_rev;
    int oriented;
    uint64_t ins;
};

static void up_visit(void* c_, uint64_t q, uint64_t i, uint64_t key, int fwd)
{
    (void)q, (void)i;
    struct up_ctx* c = c_;
    orc_table* t = c->t;
    uint64_t* p = slot_of(t, key);
    uint64_t* v = &t->val[p - t->key];
    const uint64_t x = c->oriented ? (fwd ? c->x : c->x_rev) : c->x;
    if(*p == EMPTY)
    {
        *p = key;
        /* Absent: the value given, or f(T(), fwd) when oriented (Streaming_Kmer_Hash_Table.hpp:682, 2292-2295). */
        *v = c->oriented ? apply(t, c->op, 0, x) : (c->init & t->vmask);
        t->n++;
        c->ins++;
        if(t->n * 2 > t->slots)
            grow(t);
        return;
    }
    *v = apply(t, c->op, *v, x);
}

uint64_t orc_upsert(orc_table* t, const uint32_t user, const char* bases, const uint64_t* off, const uint64_t n, const uint32_t op, const uint64_t x, const uint64_t init)
{
    struct up_ctx c = {t, op, x, init, 0, 0, 0};
    stream(t->k, bases, off, n, up_visit, &c);
    account(t, user, c.ins);
    return c.ins;
}

uint64_t orc_upsert_oriented(orc_table* t, const uint32_t user, const char* bases, const uint64_t* off, const uint64_t n, const uint32_t op, const uint64_t x_fwd, const uint64_t x_rev)
{
    struct up_ctx c = {t, op, x_fwd, 0, x_rev, 1, 0};
    stream(t->k, bases, off, n, up_visit, &c);
    account(t, user, c.ins);
    return c.ins;
}

struct upd_ctx { orc_table* t; uint32_t op; uint64_t x, found; };

static void upd_visit(void* c_, uint64_t q, uint64_t i, uint64_t key, int fwd)
{
    (void)q, (void)i, (void)fwd;
    struct upd_ctx* c = c_;
    uint64_t* p = slot_of(c->t, key);
    if(*p == EMPTY)
        return;
    uint64_t* v = &c->t->val[p - c->t->key];
    *v = apply(c->t, c->op, *v, c->x);
    c->found++;
}

uint64_t orc_update(orc_table* t, const char* bases, const uint64_t* off, const uint64_t n, const uint32_t op, const uint64_t x)
{
    struct upd_ctx c = {t, op, x, 0};
    stream(t->k, bases, off, n, upd_visit, &c);
    return c.found;
}

struct look_ctx
{
    const orc_table* t;
    const uint64_t* pos_off;
    uint8_t* found;
    uint64_t* values;
    uint8_t* fwd;
    uint64_t* counts;
    uint64_t m_fwd, m_rev;
    int mode; /* 0 lookup, 1 count, 2 count_masked, 3 sum */
};

static void look_visit(void* c_, uint64_t q, uint64_t i, uint64_t key, int fwd)
{
    struct look_ctx* c = c_;
    const uint64_t* p = slot_of(c->t, key);
    const int hit = (*p != EMPTY);
    const uint64_t v = hit ? c->t->val[p - c->t->key] : 0;
    switch(c->mode)
    {
    case 0:
    {
        const uint64_t j = c->pos_off[q] + i;
        c->found[j] = hit ? 1 : 0;
        if(c->values)
            c->values[j] = v;
        if(c->fwd)
            c->fwd[j] = (uint8_t)fwd;
        break;
    }
    case 1: c->counts[q] += hit; break;
    case 2: c->counts[q] += hit && (v & (fwd ? c->m_fwd : c->m_rev)) != 0; break;
    default: c->counts[q] += v; break;
    }
}

void orc_lookup(const orc_table* t, const char* bases, const uint64_t* off, const uint64_t n, uint8_t* found, uint64_t* values, uint8_t* fwd)
{
    /* Output offsets o_i = the positions of the sequences before it (capi/Kmer_Table.hpp:165-168). */
    uint64_t* o = malloc((n + 1) * sizeof(uint64_t));
    uint64_t p = 0;
    for(uint64_t i = 0; i < n; ++i)
    {
        const uint64_t len = off[i + 1] - off[i];
        o[i] = p, p += len >= (uint64_t)t->k ? len - t->k + 1 : 0;
    }
    memset(found, 2, p);
    if(values)
        memset(values, 0, p * sizeof(uint64_t));
    if(fwd)
        memset(fwd, 0, p);
    struct look_ctx c = {t, o, found, values, fwd, NULL, 0, 0, 0};
    stream(t->k, bases, off, n, look_visit, &c);
    free(o);
}

void orc_count(const orc_table* t, const char* bases, const uint64_t* off, const uint64_t n, uint64_t* counts)
{
    memset(counts, 0, n * sizeof(uint64_t));
    struct look_ctx c = {t, NULL, NULL, NULL, NULL, counts, 0, 0, 1};
    stream(t->k, bases, off, n, look_visit, &c);
}

void orc_count_masked(const orc_table* t, const char* bases, const uint64_t* off, const uint64_t n, const uint64_t m_fwd, const uint64_t m_rev, uint64_t* counts)
{
    memset(counts, 0, n * sizeof(uint64_t));
    struct look_ctx c = {t, NULL, NULL, NULL, NULL, counts, m_fwd & t->vmask, m_rev & t->vmask, 2};
    stream(t->k, bases, off, n, look_visit, &c);
}

void orc_sum(const orc_table* t, const char* bases, const uint64_t* off, const uint64_t n, uint64_t* sums)
{
    memset(sums, 0, n * sizeof(uint64_t));
    struct look_ctx c = {t, NULL, NULL, NULL, NULL, sums, 0, 0, 3};
    stream(t->k, bases, off, n, look_visit, &c);
}

/* Streaming_Kmer_Hash_Table.hpp:2608-2645: absent unless the first k characters are ACGT. */
int orc_get(const orc_table* t, const char* kmer, uint64_t* value)
{
    uint64_t f = 0;
    for(int i = 0; i < t->k; ++i)
    {
        if(!is_acgt(kmer[i]))
        {
            *value = 0;
            return 0;
        }
        f = (f << 2) | code(kmer[i]);
    }
    const uint64_t r = orc_revcomp(f, t->k), key = f < r ? f : r;
    const uint64_t* p = slot_of(t, key);
    if(*p == EMPTY)
    {
        *value = 0;
        return 0;
    }
    *value = t->val[p - t->key];
    return 1;
}

uint64_t orc_size(const orc_table* t) { return t->n; }
uint64_t orc_capacity(const orc_table* t) { return t->cap * B; }

static int cmp_u64(const void* a, const void* b)
{
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : x > y;
}

uint64_t orc_dump(const orc_table* t, uint64_t* keys, uint64_t* values)
{
    uint64_t c = 0;
    for(uint64_t i = 0; i < t->slots; ++i)
        if(t->key[i] != EMPTY)
            keys[c++] = t->key[i];
    qsort(keys, c, sizeof(uint64_t), cmp_u64);
    if(values)
        for(uint64_t i = 0; i < c; ++i)
            values[i] = t->val[slot_of(t, keys[i]) - t->key];
    return c;
}

/* capi/Kmer_Table.hpp:203-230. */
uint64_t orc_reduce(const orc_table* t, const uint32_t what, uint64_t mask)
{
    mask &= t->vmask;
    uint64_t r = 0;
    for(uint64_t i = 0; i < t->slots; ++i)
    {
        if(t->key[i] == EMPTY)
            continue;
        const uint64_t v = t->val[i] & mask;
        if(t->vb == 0)
            r++;
        else if(what == 0)
            r += v != 0;
        else if(what == 1)
            r += (uint64_t)__builtin_popcountll(v);
        else
            r += v;
    }
    return r;
}

/* counter/Kmer_Set_Counter.cpp:96-119. */
void orc_histogram(const orc_table* t, const uint64_t max, uint64_t* h)
{
    memset(h, 0, (max + 1) * sizeof(uint64_t));
    for(uint64_t i = 0; i < t->slots; ++i)
        if(t->key[i] != EMPTY && t->val[i] >= 1 && t->val[i] <= max)
            h[t->val[i]]++;
}

/* The capacity (in slots) after each of a single user's calls that inserted ins[0..calls) keys, into a table sized
 * for max_sz keys: the schedule of account() alone, for checking capacities at sizes the exact dictionary would not
 * hold. */
void orc_replay_capacity(const uint64_t max_sz, const double lf, const int pow2, const uint64_t* ins, const uint64_t calls, uint64_t* caps)
{
    orc_table t;
    memset(&t, 0, sizeof(t));
    t.lf = lf;
    t.cap = orc_cap_for(max_sz, lf, pow2);
    t.resize_th = (uint64_t)((double)(t.cap * B) * lf);
    t.step = step_for(t.resize_th);
    for(uint64_t i = 0; i < calls; ++i)
    {
        account(&t, 0, ins[i]);
        caps[i] = t.cap * B;
    }
}

/* Stafford's variant-13 finaliser, for the digest below. */
static uint64_t dig_mix(uint64_t x)
{
    x ^= x >> 30, x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27, x *= 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

/* An order-independent digest of a multiset of (key, value) pairs, for comparing dumps too large to sort in a test:
 * out[0] the pair count, out[1] and out[2] sums modulo 2^64 of two unrelated 64-bit mixes of each pair. Dumps of the
 * same pairs in any order give the same digest; different ones agree only by chance. values may be NULL (a set). */
void orc_digest(const uint64_t* keys, const uint64_t* values, const uint64_t n, uint64_t* out)
{
    uint64_t a = 0, b = 0;
    for(uint64_t i = 0; i < n; ++i)
    {
        const uint64_t v = values ? values[i] : 0;
        a += dig_mix(keys[i] ^ dig_mix(v + 0x632BE59BD9B4E019ull));
        b += dig_mix((keys[i] + 0x9E3779B97F4A7C15ull) * 0xD1342543DE82EF95ull ^ dig_mix(v ^ 0x3C6EF372FE94F82Aull));
    }
    out[0] = n, out[1] = a, out[2] = b;
}
