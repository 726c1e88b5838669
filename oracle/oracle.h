/* CPU restatement of kache-hash's streaming k-mer table semantics: the checker for the CUDA path.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load this
 * library, and only to check or to time a baseline; the product never links, loads or calls it.
 *
 * What it restates (file:line of the reference, kache-hash v0.7.1):
 *   - the describers' k-mer descriptions: 2-bit codes (Kmer_Batch.hpp:108), canonical forms and orientation
 *     (Kmer_Batch.hpp:230-241), Wang's hash (Kmer_Batch.hpp:24-35), checksums (Kmer_Batch.hpp:44-67, the
 *     non-AVX-512 variant), l-minimizer hashes (Kmer_Batch.hpp:204-227, Kmer_Lanes.hpp:247-274);
 *   - ACGT splitting (DNA_Utility.hpp:199-224, Streaming_Kmer_Hash_Table.hpp:1697-1709);
 *   - sizing: cap_for (Streaming_Kmer_Hash_Table.hpp:1004-1011), fits (:800-804), the resize threshold and the
 *     per-user flush schedule that decides when a table doubles (:383, :2244-2286, :1447-1455, :1679-1680);
 *   - the observable results of every operation: upsert / insert / upsert_oriented (:2219-2514), update
 *     (:2650-2691), find / count (:2519-2604, :2695-2700), single-k-mer find (:2608-2645), for_each (:2705-2725),
 *     and the C interface's ops, lookups and reductions (capi/Kmer_Table.hpp:30-61,134-230).
 * Placement (buckets, secondaries, the overflow table) is not observable and is not modelled: a key maps to
 * its value in one exact dictionary, processed in stream order (sequences in order, positions in order).
 */
#ifndef KACHE_ORACLE_H
#define KACHE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_KEEP = 0, ORC_ASSIGN = 1, ORC_ADD = 2, ORC_OR = 3, ORC_MIN = 4, ORC_MAX = 5, ORC_ADD_WRAP = 16 };

uint64_t orc_wang(uint64_t x);
uint8_t orc_checksum(uint64_t key);
uint64_t orc_revcomp(uint64_t x, int k);
uint64_t orc_minimizer_hash(uint64_t key, int k, int l);

/* Describes the len-k+1 positions of s: canonical key, minimizer hash, checksum, orientation (1 iff the k-mer
 * occurs as its canonical form), validity (0 iff a non-ACGT character lies in it; then the rest are 0).
 * Returns the number of positions. */
uint64_t orc_describe(const char* s, uint64_t len, int k, int l, uint64_t* key, uint64_t* h, uint8_t* cs, uint8_t* fwd, uint8_t* valid);

uint64_t orc_cap_for(uint64_t max_sz, double lf, int pow2);
void orc_replay_capacity(uint64_t max_sz, double lf, int pow2, const uint64_t* ins, uint64_t calls, uint64_t* caps);
int orc_fits(uint64_t max_sz, double lf, int pow2);

typedef struct orc_table orc_table;

orc_table* orc_new(int k, int value_bytes, uint64_t max_sz, double lf, int pow2);
void orc_free(orc_table* t);
uint32_t orc_register(orc_table* t);

/* Batches: sequences concatenated in `bases`, sequence i at [off[i], off[i+1]). */
uint64_t orc_upsert(orc_table* t, uint32_t user, const char* bases, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x, uint64_t init);
uint64_t orc_upsert_oriented(orc_table* t, uint32_t user, const char* bases, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x_fwd, uint64_t x_rev);
uint64_t orc_update(orc_table* t, const char* bases, const uint64_t* off, uint64_t n, uint32_t op, uint64_t x);
/* found: 0 absent, 1 present, 2 not a k-mer; at pos_off[q] + i. values and fwd may be NULL. */
void orc_lookup(const orc_table* t, const char* bases, const uint64_t* off, uint64_t n, uint8_t* found, uint64_t* values, uint8_t* fwd);
void orc_count(const orc_table* t, const char* bases, const uint64_t* off, uint64_t n, uint64_t* counts);
void orc_count_masked(const orc_table* t, const char* bases, const uint64_t* off, uint64_t n, uint64_t m_fwd, uint64_t m_rev, uint64_t* counts);
void orc_sum(const orc_table* t, const char* bases, const uint64_t* off, uint64_t n, uint64_t* sums);
int orc_get(const orc_table* t, const char* kmer, uint64_t* value);
uint64_t orc_size(const orc_table* t);
uint64_t orc_capacity(const orc_table* t);
/* Sorted dump of (key, value); returns the number of keys. */
uint64_t orc_dump(const orc_table* t, uint64_t* keys, uint64_t* values);
uint64_t orc_reduce(const orc_table* t, uint32_t what, uint64_t mask);
void orc_histogram(const orc_table* t, uint64_t max, uint64_t* h);
/* Order-independent digest of (key, value) pairs: out[0] the count, out[1..2] two sums of unrelated mixes; values may
 * be NULL. For comparing dumps too large to sort. */
void orc_digest(const uint64_t* keys, const uint64_t* values, uint64_t n, uint64_t* out);

#ifdef __cplusplus
}
#endif

#endif
