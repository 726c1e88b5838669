/* Failure injection for the tests of the B200 kache-hash library (no counterpart in the reference, whose failure
 * paths are exceptions thrown on the host).
 *
 * Two failures that a live system meets rarely, made on demand from the host so that tests can check how the library
 * answers them without faulting or hanging the GPU:
 *   - an allocation that fails: the library's next device or page-locked allocations fail as out of memory would,
 *     and the call making them returns KACHE_ENOMEM;
 *   - an insert that never publishes: a key's slot is claimed and left unpublished, as by an inserter that stopped
 *     midway, and the kernels' bounded wait for it is shortened, so that a later insert of that key whose operation
 *     must see the value first (KACHE_ASSIGN, KACHE_MIN) gives up after `wait_polls` polls and its call returns
 *     KACHE_EINTERNAL. The table is not usable afterwards: free it.
 * Not for production use. */
#ifndef KACHE_B200_TESTING_H
#define KACHE_B200_TESTING_H

#include "kache_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The `after`-th next device or page-locked allocation of the library (0: the next one) fails as out of memory; the
 * ones before it succeed, and injection is off again after it. A negative `after` turns injection off. Process-wide. */
int kache_b200_testing_fail_allocation(int64_t after) KACHE_NOEXCEPT;

/* Claims, and leaves unpublished, the slot of the canonical form of the k-mer of the table's k characters at `kmer`
 * in its primary bucket, and sets the bound of the table's waits for a racing insert to `wait_polls` polls.
 * KACHE_EINVAL if the k-mer has a non-ACGT character, is already in the table or its primary bucket is full. */
int kache_b200_testing_plant_claim(kache_table* t, const char* kmer, uint32_t wait_polls) KACHE_NOEXCEPT;

#ifdef __cplusplus
}
#endif

#endif
