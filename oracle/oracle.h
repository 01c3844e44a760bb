/*
 * oracle.h -- CPU restatement of the ops-collections bulk-container algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.  Nothing in the product links or calls it.
 *
 * Every function is a sequential, single-threaded restatement of the
 * reference's per-key algorithm, cited by file:line of the reference project.
 * Pinned by tests/golden/ (known answers from the reference's own tests plus
 * outputs of the reference's host headers, compiled where the reference
 * project is mounted by oracle/ref_probe/).
 */
#ifndef B2CO_ORACLE_H
#define B2CO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- hashes (include/detail/hash_functions/ headers) ------------------- */
uint32_t orc_xxh32(const void* bytes, size_t len, uint32_t seed);
uint64_t orc_xxh64(const void* bytes, size_t len, uint64_t seed);
uint32_t orc_murmur3_32(const void* bytes, size_t len, uint32_t seed);
uint32_t orc_fmix32(uint32_t key, uint32_t seed);
uint64_t orc_fmix64(uint64_t key, uint64_t seed);

/* Probe-hash selector, shared with include/b2co.h (B2CO_HASH_*). */
enum { ORC_HASH_XXH32 = 0, ORC_HASH_MURMUR3_32 = 1, ORC_HASH_FMIX = 2, ORC_HASH_XXH64 = 3 };
enum { ORC_PROBE_LINEAR = 0, ORC_PROBE_DOUBLE = 1 };

/* 32-bit probe hash of a key's object representation (key_bytes 2, 4 or 8;
 * the Fmix family needs 4 or 8). */
uint32_t orc_probe_hash(int hash_kind, uint64_t key_bits, uint32_t key_bytes, uint32_t seed);

/* ---- capacity (include/detail/extent/extent.inl:20-62, utility/prime.h) */
/* Number of entries of the capacity prime table and its i-th entry. */
uint64_t orc_prime_table_size(void);
uint64_t orc_prime_table_entry(uint64_t i);
/* Smallest table prime >= n; 0 when n exceeds the table's last entry. */
uint64_t orc_prime_at_least(uint64_t n);
/* Valid capacity for a request; 0 on "Invalid input Extent". */
uint64_t orc_valid_capacity(uint64_t request, uint32_t bucket_size, int probing);

/* ---- probing (include/detail/probing_scheme/probing_scheme_impl.inl) --- */
typedef struct {
    uint32_t idx, step, upper;
} orc_probe_iter;
orc_probe_iter orc_make_iter(int probing, int hash_kind, uint64_t key_bits, uint32_t key_bytes,
                             uint32_t bucket_size, uint32_t capacity);
uint32_t orc_iter_next(orc_probe_iter* it);

/* ---- open-addressing table (detail/open_addressing/open_addressing_ref_impl.h) */
typedef struct {
    uint8_t* slots;          /* capacity * slot_bytes bytes, owned by the caller */
    uint32_t capacity;
    uint32_t key_bytes;      /* 2, 4 or 8 */
    uint32_t value_bytes;    /* 0 (set), 2, 4 or 8 */
    uint32_t slot_bytes;     /* 2, 4, 8 or 16 */
    uint32_t value_offset;
    uint32_t bucket_size;
    int probing;
    int hash_kind;
    uint64_t empty_key;
    uint64_t empty_value;
    uint64_t erased_key;     /* == empty_key when no tombstone is configured */
    int key_kind;            /* ORC_KEY_INT: bitwise key match; ORC_KEY_FLOAT: IEEE == (fp16/fp32/fp64) */
} orc_table;

/* Key kinds: the reference matches keys with KeyEqual (==, utility/equal_wrapper.h:30-33)
 * and tests sentinels bitwise (:35-42; utility/traits.h:27-28). */
enum { ORC_KEY_INT = 0, ORC_KEY_FLOAT = 1 };

/* KeyEqual of a table of this key kind on two key bit patterns. */
int orc_key_equal(int key_kind, uint32_t key_bytes, uint64_t a, uint64_t b);

/* Slot layout of Pair<K,V> (pair.inl:19-24) or of a bare key. */
void orc_slot_layout(uint32_t key_bytes, uint32_t value_bytes, uint32_t* slot_bytes, uint32_t* value_offset);
void orc_table_clear(orc_table* t);

enum { ORC_FAILED = 0, ORC_SUCCESS = 1, ORC_DUPLICATE = 2 };

/* Bulk forms; inputs are packed little-endian keys (key_bytes each) and values
 * (value_bytes each).  All run sequentially in input order. */
uint64_t orc_insert(orc_table* t, const void* keys, const void* values, const uint8_t* stencil, uint64_t n);
uint64_t orc_insert_or_assign(orc_table* t, const void* keys, const void* values, uint64_t n,
                              uint64_t* assigned);
void orc_assign_if(orc_table* t, const void* keys, const void* values, const uint8_t* stencil, uint64_t n);
void orc_insert_and_find(orc_table* t, const void* keys, const void* values, uint64_t n, void* out_found,
                         uint8_t* out_inserted);
void orc_find(const orc_table* t, const void* keys, const uint8_t* stencil, uint64_t n, void* out_values,
              uint32_t* out_windows);
void orc_contains(const orc_table* t, const void* keys, const uint8_t* stencil, uint64_t n, uint8_t* out,
                  uint32_t* out_windows);
/* Multi-threaded (OpenMP) read-only Find and Contains: the timed CPU baseline
 * and the checker of full-size query streams. */
void orc_find_parallel(const orc_table* t, const void* keys, uint64_t n, void* out_values, int threads);
void orc_contains_parallel(const orc_table* t, const void* keys, uint64_t n, uint8_t* out, int threads);
/* Stored-set comparison: every occupied slot of `a` (whose keys are distinct,
 * e.g. the oracle's own table) is looked up in `b`; *mismatches counts keys
 * that `b` misses or holds with another payload, *occupied_a / *occupied_b
 * count the occupied (non-empty, non-tombstone) slots.  The two stored pair
 * sets are equal exactly when mismatches == 0 and the counts agree. */
void orc_pairs_match(const orc_table* a, const orc_table* b, uint64_t* occupied_a, uint64_t* occupied_b,
                     uint64_t* mismatches, int threads);
/* Many independent tables (the batched pattern): table i has capacity caps[i]
 * (valid, slots in `slab` from slot offset slot_off[i]), inserts pairs
 * [ins_off[i], ins_off[i+1]) of keys/values in order, then answers queries
 * [q_off[i], q_off[i+1]).  Each table is rebuilt sequentially by the oracle
 * (tables in parallel), its stored set compared with the slab's segment (the
 * device's tables), and its Find results written to out_expected.  Returns the
 * number of tables whose stored set differs; the first one goes to *first_bad. */
uint64_t orc_group_check(uint64_t count, const uint64_t* caps, const uint64_t* slot_off, const uint8_t* slab,
                         const orc_table* shape, const void* keys, const void* values, const uint64_t* ins_off,
                         const void* queries, const uint64_t* q_off, void* out_expected, uint64_t* first_bad,
                         int threads);
uint64_t orc_erase(orc_table* t, const void* keys, uint64_t n);
uint64_t orc_count(const orc_table* t, const void* keys, uint64_t n);

/* ---- Bloom filter (bloom_filter_policy.h:99-178, bloom_filter_impl.h:40-80) */
/* Any BloomFilterPolicy with 32-bit words: wpb words per block, pattern_bits bits per key. */
int orc_bloom_policy_valid(uint32_t wpb, uint32_t pattern_bits);
uint32_t orc_bloom_word_pattern(uint32_t w, uint32_t bpw, uint32_t lower);
void orc_bloom_add_policy(uint32_t* words, uint64_t num_blocks, uint32_t wpb, uint32_t pattern_bits, const void* keys,
                          uint32_t key_bytes, uint64_t n, uint64_t seed);
void orc_bloom_contains_policy(const uint32_t* words, uint64_t num_blocks, uint32_t wpb, uint32_t pattern_bits,
                               const void* keys, uint32_t key_bytes, uint64_t n, uint64_t seed, uint8_t* out,
                               int threads);
/* The default policy (8 words per block, PatternBits 8). */
void orc_bloom_add(uint32_t* words, uint64_t num_blocks, const void* keys, uint32_t key_bytes, uint64_t n,
                   uint64_t seed);
void orc_bloom_contains(const uint32_t* words, uint64_t num_blocks, const void* keys, uint32_t key_bytes,
                        uint64_t n, uint64_t seed, uint8_t* out);
void orc_bloom_contains_parallel(const uint32_t* words, uint64_t num_blocks, const void* keys, uint32_t key_bytes,
                                 uint64_t n, uint64_t seed, uint8_t* out, int threads);

/* ---- HyperLogLog (hyperloglog_ref.h:30-47, hyperloglog.inl:327-345, finalizer.h) */
void orc_hll_add(uint8_t* registers, uint32_t precision, const void* keys, uint32_t key_bytes, uint64_t n);
void orc_hll_add_parallel(uint8_t* registers, uint32_t precision, const void* keys, uint32_t key_bytes, uint64_t n,
                          int threads);
void orc_hll_merge(uint8_t* dst, const uint8_t* src, uint32_t precision);
void orc_hll_histogram(const uint8_t* registers, uint32_t precision, uint32_t hist[65]);
/* Finalizer over a histogram; bias tables are supplied by the caller (the
 * oracle does not own them: they are the product's data and are pinned
 * against the reference separately). */
uint64_t orc_hll_finalize(uint32_t precision, const uint32_t hist[65], const double* raw_estimates,
                          const double* biases, int n_points, double threshold);

#ifdef __cplusplus
}
#endif
#endif
