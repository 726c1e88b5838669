/* kache-hash's C interface, served by hand-written CUDA kernels on one B200.
 *
 * Drop-in replacement for kache-hash's capi/kache_capi.h: the same functions, prototypes, enums, struct layouts and
 * status codes, so that existing callers (the Rust crate rust/kache-hash-sys/src/lib.rs:59-80, capi users) relink
 * against libkache_b200.so unchanged. Each declaration cites the reference declaration it replaces.
 *
 * A table holds canonical k-mers (the lesser of a k-mer and its reverse complement), as a set or as a map to
 * unsigned values of 1, 2, 4 or 8 bytes, in HBM. Batches of sequences come from host memory; non-ACGT characters
 * split them and lowercase bases count. Threading follows the reference's rules: inserts may run from several
 * users' threads, updates only with updates, queries only with queries (the library serialises its GPU work per
 * table). Every fallible function returns a status and catches every exception; a CUDA failure reads as
 * KACHE_EINTERNAL, a failed device or pinned allocation as KACHE_ENOMEM.
 */
#ifndef KACHE_HASH_CAPI_H
#define KACHE_HASH_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#define KACHE_NOEXCEPT noexcept
#else
#define KACHE_NOEXCEPT
#endif

/* Status codes (reference capi/kache_capi.h:34-41). */
enum
{
    KACHE_OK = 0,
    KACHE_EINVAL = 1,
    KACHE_EUSERS = 2,
    KACHE_ENOMEM = 3,
    KACHE_EINTERNAL = 4
};

/* Most users of one table (reference capi/kache_capi.h:43). */
#define KACHE_MAX_USERS 128

/* How an insert or update combines a value v with an operand x (reference capi/kache_capi.h:46-54): keep v, x,
 * v + x saturating at the width's maximum, v | x, min, max. */
enum
{
    KACHE_KEEP = 0,
    KACHE_ASSIGN = 1,
    KACHE_ADD = 2,
    KACHE_OR = 3,
    KACHE_MIN = 4,
    KACHE_MAX = 5
};

/* Reductions over all keys with a value mask m (reference capi/kache_capi.h:58-63): keys with v & m nonzero (every
 * key of a set), total popcount of v & m, sum of v & m modulo 2^64. */
enum
{
    KACHE_REDUCE_KEYS = 0,
    KACHE_REDUCE_POPCOUNT = 1,
    KACHE_REDUCE_SUM = 2
};

/* Per-position lookup results (reference capi/kache_capi.h:66-71). */
enum
{
    KACHE_ABSENT = 0,
    KACHE_PRESENT = 1,
    KACHE_NOT_KMER = 2
};

typedef struct kache_table kache_table;

/* Table options (reference capi/kache_capi.h:78-87). resize_workers is validated (>= 1) and otherwise unused: the
 * GPU resizes with its own grid. */
typedef struct kache_options
{
    uint32_t k;
    uint32_t value_bytes;
    uint64_t expected_keys;
    double load_factor;
    uint32_t resize_workers;
    uint32_t pow2_capacity;
} kache_options;

/* Table statistics (reference capi/kache_capi.h:90-99). capacity is the reference's slot count exactly; bytes and
 * the placement percentages describe this implementation's layout. */
typedef struct kache_stats
{
    uint64_t capacity;
    uint64_t bytes;
    uint64_t keys;
    uint64_t overflow_keys;
    double primary_pct;
    double secondary_pct;
    double overflow_pct;
} kache_stats;

/* Iteration callback (reference capi/kache_capi.h:106): chunks of at most 4096 keys in 2-bit encoding, first base
 * most significant; values of the table's width, NULL for a set; nonzero stops the iteration. */
typedef int (*kache_keys_fn)(void* ctx, const uint64_t* keys, const void* values, size_t n);

/* reference capi/kache_capi.h:111 */
int kache_supports(uint32_t k, uint32_t value_bytes) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:116 */
kache_options kache_default_options(uint32_t k, uint32_t value_bytes) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:120 */
int kache_new(const kache_options* options, kache_table** out) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:123 */
void kache_free(kache_table* t) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:128 */
int kache_register(kache_table* t, uint32_t* user) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:135 */
int kache_insert(kache_table* t, uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t* inserted) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:141 */
int kache_insert_oriented(kache_table* t, uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x_fwd, uint64_t x_rev, uint64_t* inserted) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:147 */
int kache_update(kache_table* t, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t* present) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:152 */
int kache_count(const kache_table* t, const char* const* seqs, const size_t* lens, size_t n, uint64_t* counts) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:159 */
int kache_count_masked(const kache_table* t, const char* const* seqs, const size_t* lens, size_t n, uint64_t mask_fwd, uint64_t mask_rev, uint64_t* counts) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:164 */
int kache_sum(const kache_table* t, const char* const* seqs, const size_t* lens, size_t n, uint64_t* sums) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:174 */
int kache_lookup(const kache_table* t, const char* const* seqs, const size_t* lens, size_t n, uint8_t* found, void* values, uint8_t* fwd) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:180 */
int kache_get(const kache_table* t, const char* kmer, uint8_t* found, uint64_t* value) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:184 */
int kache_size(const kache_table* t, uint64_t* keys) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:190 */
int kache_reduce(const kache_table* t, uint32_t what, uint64_t mask, uint32_t workers, uint64_t* out) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:196 */
int kache_for_each(const kache_table* t, uint32_t shards, uint32_t shard, kache_keys_fn f, void* ctx) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:199 */
int kache_get_stats(const kache_table* t, kache_stats* out) KACHE_NOEXCEPT;

/* reference capi/kache_capi.h:202 */
const char* kache_strerror(int code) KACHE_NOEXCEPT;

#ifdef __cplusplus
}
#endif

#endif
