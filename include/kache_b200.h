/* Extensions of the B200 kache-hash library beyond the reference's C interface.
 *
 * These expose what the reference offers only through its C++ templates (other k and l, the template API's
 * wrapping `v + x`, separate initial values; include/Streaming_Kmer_Hash_Table.hpp:624-745), its counter library
 * (counter/Kmer_Set_Counter.hpp:23-76), and what a GPU caller needs on top: batches already resident in HBM,
 * the CUDA stream to run on, and per-kernel timing. Tables made here are kache_table handles: every kache_* function
 * of kache_capi.h works on them.
 */
#ifndef KACHE_B200_H
#define KACHE_B200_H

#include "kache_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* An operation beyond the reference C interface's: v + x modulo 2^(8 * value_bytes), the template API's counting
 * functor (test/check.cpp `inc`, counter/Kmer_Set_Counter.cpp:85). */
#define KACHE_B200_ADD_WRAP 16u

/* Creates a table of k-mers with l-minimizers: (k, l) one of (31, 22), (27, 16), (32, 20); value_bytes 0, 1, 2, 4,
 * 8; sized as the reference's Streaming_Kmer_Hash_Table(expected_keys, workers, load_factor, pow2_capacity)
 * (include/Streaming_Kmer_Hash_Table.hpp:624,771-796). */
int kache_b200_new(uint32_t k, uint32_t l, uint32_t value_bytes, uint64_t expected_keys, double load_factor, uint32_t pow2_capacity, kache_table** out) KACHE_NOEXCEPT;

/* Runs the table's work on the CUDA stream `stream` (a cudaStream_t; NULL for the table's own stream). */
int kache_b200_set_stream(kache_table* t, void* stream) KACHE_NOEXCEPT;

/* upsert with the initial value `init` for absent keys and f(v) = op(v, x) for present ones, op including
 * KACHE_B200_ADD_WRAP (include/Streaming_Kmer_Hash_Table.hpp:672). In a set, an insert. */
int kache_b200_upsert(kache_table* t, uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t init, uint64_t* inserted) KACHE_NOEXCEPT;

/* upsert_oriented with op one of KACHE_ASSIGN, KACHE_ADD, KACHE_OR, KACHE_MAX, KACHE_B200_ADD_WRAP
 * (include/Streaming_Kmer_Hash_Table.hpp:682). */
int kache_b200_upsert_oriented(kache_table* t, uint32_t user, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x_fwd, uint64_t x_rev, uint64_t* inserted) KACHE_NOEXCEPT;

/* update with op including KACHE_B200_ADD_WRAP (include/Streaming_Kmer_Hash_Table.hpp:698). */
int kache_b200_update(kache_table* t, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t* present) KACHE_NOEXCEPT;

/* Batches resident in device memory: sequence i is d_bases[d_off[i], d_off[i + 1]), d_off holding n + 1 offsets.
 * Outputs of the lookups are device pointers too, laid out as kache_lookup's. Results returned by value
 * (inserted, present) are read back, so each call ends synchronised with its stream. */
int kache_b200_upsert_dev(kache_table* t, uint32_t user, const uint8_t* d_bases, const uint64_t* d_off, uint64_t n, uint32_t op, uint64_t x, uint64_t init, uint64_t* inserted) KACHE_NOEXCEPT;
int kache_b200_upsert_oriented_dev(kache_table* t, uint32_t user, const uint8_t* d_bases, const uint64_t* d_off, uint64_t n, uint32_t op, uint64_t x_fwd, uint64_t x_rev, uint64_t* inserted) KACHE_NOEXCEPT;
int kache_b200_update_dev(kache_table* t, const uint8_t* d_bases, const uint64_t* d_off, uint64_t n, uint32_t op, uint64_t x, uint64_t* present) KACHE_NOEXCEPT;
int kache_b200_lookup_dev(kache_table* t, const uint8_t* d_bases, const uint64_t* d_off, uint64_t n, uint8_t* d_found, void* d_values, uint8_t* d_fwd) KACHE_NOEXCEPT;
int kache_b200_count_dev(kache_table* t, const uint8_t* d_bases, const uint64_t* d_off, uint64_t n, uint64_t* d_counts) KACHE_NOEXCEPT;

/* Several batches resident in device memory, run as one call (no counterpart in the reference, whose callers make
 * one call per batch, benchmark/measure.cpp:45-140): their sequences share one segment list and one launch, so many
 * small batches -- a few hundred reads each -- fill the GPU as one large batch does, while each batch keeps its own
 * arrays and results. Each sequence is read where its batch holds it; nothing is copied. kind is one of
 * KACHE_B200_RUN_*; op, x and y are the operation and its operands (upsert: x and init; oriented upsert: x_fwd and
 * x_rev; update: x). Per batch, `result` is set to the keys it inserted (upserts; a key that two batches of the call
 * insert is credited to one of them), the k-mers of it present (update), its positions found (lookup: found flags
 * equal to 1) or the sum of its per-sequence counts (count). Lookups write each
 * batch's found flags, values and orientations to its out0, out1, out2 (device arrays laid out as kache_lookup's;
 * out1 and out2 may be NULL); counts write its per-sequence counts to out0 (a device array of n uint64_t). The call
 * returns synchronised with the table's stream. */
typedef struct kache_dev_batch {
    const uint8_t* d_bases;     /* sequence i is d_bases[d_off[i], d_off[i + 1]) */
    const uint64_t* d_off;      /* n + 1 offsets, in device memory */
    uint64_t n;
    void* out0;
    void* out1;
    void* out2;
    uint64_t result;
} kache_dev_batch;
#define KACHE_B200_RUN_UPSERT          0u
#define KACHE_B200_RUN_UPSERT_ORIENTED 1u
#define KACHE_B200_RUN_UPDATE          2u
#define KACHE_B200_RUN_LOOKUP          3u
#define KACHE_B200_RUN_COUNT           4u
int kache_b200_run_dev_batches(kache_table* t, uint32_t user, uint32_t kind, uint32_t op, uint64_t x, uint64_t y, kache_dev_batch* batches, size_t count) KACHE_NOEXCEPT;

/* Lookups that can be captured in a CUDA graph (no counterpart in the reference): a batch shape -- n sequences with
 * the device offsets d_off[0..n] -- is staged once by kache_b200_prepare_dev (which synchronises); then
 * kache_b200_lookup_prepared looks up any batch with those offsets (the same lengths, any bases) as ONE kernel launch
 * on the table's stream: no staging, no allocation, no synchronisation, so a caller can capture a run of them, e.g.
 * one per batch of a batch-size class, in a CUDA graph and replay it. Outputs are device arrays laid out as
 * kache_lookup's; the call returns before the lookup has run (synchronise with the table's stream, or the graph, to
 * read them). A launch captured in a graph takes the table's device arrays as they were at capture: replay it only
 * while kache_b200_table_epoch returns the value it returned at capture (upserts that grow the table, clears and
 * overflow growth move the arrays); otherwise capture again. A handle belongs to the table that made it; free it
 * (kache_b200_prepared_free) only once no launch or graph that uses it remains to run. */
typedef struct kache_prepared kache_prepared;
int kache_b200_prepare_dev(kache_table* t, const uint64_t* d_off, uint64_t n, kache_prepared** out) KACHE_NOEXCEPT;
void kache_b200_prepared_free(kache_prepared* p) KACHE_NOEXCEPT;
int kache_b200_lookup_prepared(kache_table* t, const kache_prepared* p, const uint8_t* d_bases, uint8_t* d_found, void* d_values, uint8_t* d_fwd) KACHE_NOEXCEPT;
/* Per-sequence counts of present k-mers (kache_count's) of a batch of the prepared shape, into the device array
 * d_counts[0..n): a memset and one launch on the table's stream, capturable as kache_b200_lookup_prepared is. */
int kache_b200_count_prepared(kache_table* t, const kache_prepared* p, const uint8_t* d_bases, uint64_t* d_counts) KACHE_NOEXCEPT;
int kache_b200_table_epoch(kache_table* t, uint64_t* epoch) KACHE_NOEXCEPT;

/* kache_b200_count_dev for callers that cannot allocate device memory: no counterpart in the reference.
 *
 * Callers running inside their own memory pool (whose allocator must not be re-entered) or in a process that budgets
 * every byte of HBM itself cannot let the library call cudaMalloc on a query. This entry point allocates nothing: its
 * scratch (the batch's segment list) lives in one fixed 8 MiB device array that every GPU which loads the library
 * holds until the process exits. It takes at most KACHE_B200_NOALLOC_MAX_SEGMENTS sequences and as many segments of
 * up to 512 k-mer positions; beyond that it returns KACHE_EINVAL, up front when n is over the limit, else after
 * listing the segments, in which case nothing is counted and d_counts[0..n) holds zeros. Tables of 31-mers with
 * 22-minimizers only (those of kache_new). Every call shares the array and clears its header first, so calls whose
 * GPU work overlaps (other streams or threads) race: serialise them. The first call on a device looks the array's
 * device address up (cudaGetSymbolAddress); make that first call before any stream capture. The call reads a flag
 * back from the device and returns synchronised with the table's stream. */
#define KACHE_B200_NOALLOC_MAX_SEGMENTS 1048544ull
int kache_b200_count_dev_noalloc(kache_table* t, const uint8_t* d_bases, const uint64_t* d_off, uint64_t n, uint64_t* d_counts) KACHE_NOEXCEPT;

/* The describer's output per position, laid out as kache_lookup's: canonical key, minimizer hash, checksum,
 * orientation, whether the k characters are all ACGT. For checking the describer against the reference's. */
int kache_b200_describe(kache_table* t, const char* const* seqs, const size_t* lens, size_t n, uint64_t* key, uint64_t* h, uint8_t* cs, uint8_t* fwd, uint8_t* valid) KACHE_NOEXCEPT;

/* The histogram of values in [1, max] into h[0..max] (h[0] = 0) (counter/Kmer_Set_Counter.cpp:96-119). */
int kache_b200_histogram(kache_table* t, uint64_t max, uint64_t* h) KACHE_NOEXCEPT;

/* Empties the table: no keys, the capacity it was created with, every user's pending count at 0; registered users
 * stay registered. */
int kache_b200_clear(kache_table* t) KACHE_NOEXCEPT;

/* Device time and launch count of the table's kernels of one kind since profiling was switched on, measured with
 * CUDA events recorded around each launch on the table's stream. Kinds: 0 upsert, 1 update, 2 lookup, 3 per-sequence
 * reductions, 4 resize, 5 everything else. */
int kache_b200_profile(kache_table* t, int on) KACHE_NOEXCEPT;
int kache_b200_profile_read(kache_table* t, uint32_t kind, double* ms, uint64_t* launches) KACHE_NOEXCEPT;

/* Kernels this library has launched in this process, over all tables. */
uint64_t kache_b200_kernel_launches(void) KACHE_NOEXCEPT;

/* The current device's memory roofs over an array of `bytes` (rounded down to a power of 2; at least 1 MiB), as the
 * reference's roof tool measures the host's (tools/memory-roof.cpp:21-29). kind 0: sequential reads, *rate in
 * bytes/s; 1: independent random reads of 32-byte sectors, *rate in sectors/s; 2: independent random atomic adds,
 * one per sector, *rate in updates/s; 3: dependent random reads (a pointer chase over sectors by one warp per SM, so
 * nearly unloaded), *rate in loads/s over those threads. `accesses` sets the random kinds' work; *ms is the timed launch's duration. Allocates and frees the
 * array itself. */
int kache_b200_memory_roof(uint64_t bytes, uint32_t kind, uint64_t accesses, double* ms, double* rate) KACHE_NOEXCEPT;

/* A request server over a table (no counterpart in the reference, whose callers share a table through user tokens):
 * requests submitted from any threads are run by one dispatcher thread, which merges the requests waiting when the
 * GPU frees up into one call: the oldest waiting request and all waiting requests of its kind (and, for upserts,
 * the same op, x and init) whose staging fits `budget_bytes` (0: no limit beyond half the device memory free at
 * creation). Requests of one kind run in submission order; waiting requests of different kinds are concurrent (wait
 * for a request before submitting one that must see it). Runs never overlap, so queries never overlap inserts. A request's sequences and output arrays must stay valid until
 * kache_b200_server_wait returns for it. Results: an upsert's keys inserted; a lookup's found flags, values and
 * orientations as kache_lookup lays them out, and its present positions; a count's per-sequence counts as kache_count
 * lays them out, and their sum. The server registers one user of the table. */
typedef struct kache_server kache_server;
#define KACHE_B200_REQ_UPSERT 0u   /* op, x, init as kache_b200_upsert; out0..2 unused */
#define KACHE_B200_REQ_LOOKUP 1u   /* out0 found (required), out1 values (or NULL), out2 fwd (or NULL) */
#define KACHE_B200_REQ_COUNT  2u   /* out0 counts, uint64_t per sequence */
int kache_b200_server_new(kache_table* t, uint64_t budget_bytes, kache_server** out) KACHE_NOEXCEPT;
void kache_b200_server_free(kache_server* s) KACHE_NOEXCEPT;
int kache_b200_server_submit(kache_server* s, uint32_t kind, const char* const* seqs, const size_t* lens, size_t n, uint32_t op, uint64_t x, uint64_t init, void* out0, void* out1, void* out2, uint64_t* ticket) KACHE_NOEXCEPT;
/* A request whose sequences and outputs are already in device memory, laid out as kache_b200_run_dev_batches's
 * batches: sequence i is d_bases[d_off[i], d_off[i + 1]), outputs out0..2 are device arrays as kache_b200_server_submit
 * takes them. The arrays must hold their data when submitted (the work writing them finished) and stay valid until
 * kache_b200_server_wait returns for it. Device requests merge only with device requests of the same kind (and, for
 * upserts, op, x and init), into one kache_b200_run_dev_batches call: nothing is gathered or copied on the host. Their
 * results are those of host requests: keys inserted, positions found, or the sum of the counts. */
int kache_b200_server_submit_dev(kache_server* s, uint32_t kind, const uint8_t* d_bases, const uint64_t* d_off, uint64_t n, uint32_t op, uint64_t x, uint64_t init, void* out0, void* out1, void* out2, uint64_t* ticket) KACHE_NOEXCEPT;
/* Waits for a request; its result at *result, the time from its submission to its completion at *latency_ms. */
int kache_b200_server_wait(kache_server* s, uint64_t ticket, uint64_t* result, double* latency_ms) KACHE_NOEXCEPT;
/* Merged runs so far, and the requests they ran. */
int kache_b200_server_stats(kache_server* s, uint64_t* runs, uint64_t* requests) KACHE_NOEXCEPT;

/* Reads the FASTA or FASTQ file (or pipe) at `path` and calls f(ctx, seqs, lens, n) with its non-empty sequences in
 * order, in batches of whole sequences of about `batch_bases` bases, until f returns nonzero
 * (counter/Fastx_Reader.hpp:13-52). Unreadable, gzip-compressed or malformed input returns KACHE_EINVAL. */
typedef int (*kache_seqs_fn)(void* ctx, const char* const* seqs, const size_t* lens, size_t n);
int kache_b200_fastx_read(const char* path, uint64_t batch_bases, kache_seqs_fn f, void* ctx) KACHE_NOEXCEPT;

/* The counter library (counter/Kmer_Set_Counter.hpp:23-76): a set of 31-mers primed at count 0 and counted by
 * present-only increments that wrap at 2^32. Paths name FASTA or FASTQ files, or pipes. */
typedef struct kache_counter kache_counter;
int kache_counter_new(uint32_t k, uint64_t n, uint32_t threads, double load_factor, kache_counter** out) KACHE_NOEXCEPT;
void kache_counter_free(kache_counter* c) KACHE_NOEXCEPT;
int kache_counter_prime(kache_counter* c, const char* path) KACHE_NOEXCEPT;
int kache_counter_count(kache_counter* c, const char* path, uint64_t* found) KACHE_NOEXCEPT;
int kache_counter_prime_batch(kache_counter* c, const char* const* seqs, const size_t* lens, size_t n) KACHE_NOEXCEPT;
int kache_counter_count_batch(kache_counter* c, const char* const* seqs, const size_t* lens, size_t n, uint64_t* found) KACHE_NOEXCEPT;
int kache_counter_histogram(kache_counter* c, uint64_t max, uint64_t* h) KACHE_NOEXCEPT;
int kache_counter_count_of(kache_counter* c, const char* kmer, uint64_t* count) KACHE_NOEXCEPT;
int kache_counter_size(kache_counter* c, uint64_t* n) KACHE_NOEXCEPT;
/* The counter's table, for the kache_* queries (do not free it). */
kache_table* kache_counter_table(kache_counter* c) KACHE_NOEXCEPT;

#ifdef __cplusplus
}
#endif

#endif
