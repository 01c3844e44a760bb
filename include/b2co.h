/*
 * b2co.h -- C ABI of the B200 bulk-container library (libb2co.so).
 *
 * This is the drop-in boundary for the ops-collections bulk-container hot
 * path.  The reference's boundary is its header-only C++ class-template API
 * (StaticMap, StaticSet, DynamicMap, BloomFilter, HyperLogLog); every entry
 * point below replaces one of those methods and cites it as
 * `reference: <file>:<line>`.  The C++ mirror of the class templates lives in
 * include/b2co/ and is a thin layer over these functions.
 *
 * Conventions (all from the reference's host layer):
 *   - every function returns a b2co_status; the message of the last failure on
 *     the calling thread is available from b2co_last_error();
 *   - data pointers are caller-owned DEVICE pointers unless a name says
 *     "host"; "pairs" are arrays of the table's slot type (Pair<K,V>, aligned
 *     to min(16, bitceil(sizeof K + sizeof V)); a bare key for sets);
 *   - stencils are device uint8 arrays; a nonzero byte selects the item (the
 *     C ABI carries the `u8 != 0` predicate; AlwaysTrue is a NULL stencil);
 *   - `*_async` calls are stream-ordered and return after the launch; the
 *     other calls synchronize the stream, like the reference's sync methods;
 *   - n == 0 is a no-op; a NULL data pointer with n > 0 makes a sync Insert
 *     report all n items as failed and an async call a no-op, exactly as
 *     detail/open_addressing/open_addressing_impl.h:176-201 does;
 *   - batches beyond the 32-bit index range fail with B2CO_ERANGE
 *     (open_addressing_impl.h:534-545 throws std::length_error).
 */
#ifndef B2CO_H
#define B2CO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* b2co_stream; /* a cudaStream_t; NULL = legacy default stream */

typedef enum {
    B2CO_OK = 0,
    B2CO_EINVAL = 1,   /* std::invalid_argument in the reference */
    B2CO_ERANGE = 2,   /* std::length_error */
    B2CO_ENOMEM = 3,   /* std::bad_alloc */
    B2CO_ECUDA = 4,    /* std::runtime_error: a CUDA call failed */
    B2CO_ETIMEOUT = 5, /* a bounded device-side wait expired (no reference counterpart) */
    B2CO_ELOGIC = 6,   /* std::logic_error: moved-from / storage-less object */
    B2CO_EOVERFLOW = 7 /* std::overflow_error: a result cannot be represented */
} b2co_status;

typedef enum { B2CO_HASH_XXH32 = 0, B2CO_HASH_MURMUR3_32 = 1, B2CO_HASH_FMIX = 2, B2CO_HASH_XXH64 = 3 } b2co_hash;
typedef enum { B2CO_PROBE_LINEAR = 0, B2CO_PROBE_DOUBLE = 1 } b2co_probing;
typedef enum {
    B2CO_IAF_RACE = 0,       /* reference semantics: concurrent duplicates race for the slot */
    B2CO_IAF_FIRST_WINS = 1  /* deterministic: the first occurrence in input order wins */
} b2co_iaf_mode;

/* Message of the last failed call on this thread ("" if none). */
const char* b2co_last_error(void);
const char* b2co_status_string(int status);
/* Library version string. */
const char* b2co_version(void);
/* Device wait policy (no reference counterpart).  Kernels that wait on their
 * own asynchronous copies give up after `limit_ns` (0 = the default, 1 s),
 * record it in the object's status word and return; the next synchronizing
 * call on that object reports B2CO_ETIMEOUT.  `probe_timeout` != 0 is a test
 * hook: the first wait of each block is made on a barrier that nothing ever
 * arrives on, so the timeout path runs without any fault. */
int b2co_debug_set_wait(uint64_t limit_ns, int probe_timeout);
/* Context-wide hint of the bytes the L2 fetches from DRAM per miss (32, 64 or
 * 128; 0 = only read the current value into *applied).  Random bucket windows
 * use a fraction of a 128-byte line, so a smaller granularity cuts the DRAM
 * traffic of lookups.  It applies to the calling process's whole CUDA context
 * on the current device (not to the GPU beyond the process), so it is the
 * application's choice; the library never sets it on its own.  No reference
 * counterpart. */
int b2co_set_l2_fetch_granularity(uint32_t bytes, uint64_t* applied);

/* ===================================================================== */
/* Open-addressing tables: StaticMap<K,T> and StaticSet<K>                 */
/* ===================================================================== */

/* How keys compare (KeyEqual): the reference's default EqualTo is ==
 * (utility/math_utils.h:66-70, applied by utility/equal_wrapper.h:30-33).  For
 * integer keys that is bit equality; for floating-point keys it is IEEE
 * equality, so -0.0 matches +0.0 and a NaN matches nothing.  Empty and erased
 * sentinels are always compared bitwise (equal_wrapper.h:35-42,
 * utility/traits.h:27-28), and hashes read the key's bytes, so -0.0 and +0.0
 * start different probe sequences exactly as in the reference. */
typedef enum {
    B2CO_KEY_INTEGER = 0, /* integer keys of 2, 4 or 8 bytes (int16/uint16/int32/uint32/int64/uint64) */
    B2CO_KEY_FLOAT = 1    /* fp16 (2 bytes), float (4) or double (8) keys */
} b2co_key_kind;

typedef struct {
    uint32_t key_bytes;        /* 2, 4 or 8 */
    uint32_t value_bytes;      /* 0 = StaticSet, else 2, 4 or 8 (2 only with 2-byte keys) */
    uint32_t bucket_size;      /* Storage<B>: 1, 2, 4, 5 or 8 */
    uint32_t probing;          /* b2co_probing */
    uint32_t hash;             /* b2co_hash used by the probing scheme (Fmix: 4- or 8-byte keys) */
    uint32_t key_kind;         /* b2co_key_kind (0 = integer keys) */
    uint64_t empty_key_bits;   /* sentinel bit patterns (low key_bytes / value_bytes bytes) */
    uint64_t empty_value_bits;
    uint64_t erased_key_bits;  /* tombstone key; equal to empty_key_bits = no tombstone */
} b2co_oa_desc;

typedef struct b2co_oa_table b2co_oa_table;

/* The kernels' key primitives evaluated on the host (the same source as the
 * device code), so callers and tests can check them without a GPU.
 * b2co_probe_hash: the 32-bit probe hash of a key's bytes.
 * reference: detail/hash_functions/xxhash.h:52-326, murmurhash3.h:20-106,
 * utils.h:42-66, utility/math_utils.h:14-24 (SanitizeHash).
 * b2co_key_equal: the key comparison of a table of that key kind.
 * reference: utility/equal_wrapper.h:30-33, utility/math_utils.h:66-70. */
int b2co_probe_hash(uint32_t hash, uint32_t key_bytes, uint64_t key_bits, uint32_t seed, uint32_t* out);
int b2co_key_equal(uint32_t key_kind, uint32_t key_bytes, uint64_t a_bits, uint64_t b_bits, int* equal);

/* Capacity the table gets for a requested slot count.
 * reference: include/detail/extent/extent.inl:20-62 (MakeValidExtent). */
int b2co_oa_valid_capacity(uint64_t requested, uint32_t bucket_size, uint32_t probing, uint64_t* capacity);

/* Allocate and clear a table.
 * reference: include/static_map.h:78-84, include/static_set.h:73-79,
 * detail/static_map/static_map.inl:20-36, open_addressing_impl.h:69-93. */
int b2co_oa_create(const b2co_oa_desc* desc, uint64_t requested_capacity, b2co_stream stream, b2co_oa_table** out);
/* reference: StaticMap destructor (bucket_storage.h:116-119 frees the slots). */
int b2co_oa_destroy(b2co_oa_table* table);
/* reference: static_map.h:584 Capacity(). */
int b2co_oa_capacity(const b2co_oa_table* table, uint64_t* capacity);
/* Raw device slots.  reference: static_map.h:604 Data(). */
int b2co_oa_data(const b2co_oa_table* table, void** slots);
/* The table's descriptor, sentinels masked to the key / payload widths and the
 * current erased key included: what device code compiled by the caller needs
 * to walk the slots (ForEach in include/b2co/for_each.cuh).  The reference's
 * containers expose the same through their template parameters and
 * constructor arguments (static_map.h:78-84). */
int b2co_oa_describe(const b2co_oa_table* table, b2co_oa_desc* desc);
/* Measurement aid (no reference counterpart): `n` (<= 2^31) reads of whole
 * bucket windows at pseudo-random bucket starts (`seed`) of the table's own
 * slots (16- or 8-byte), four lanes per window, nothing written.  Timing it
 * gives the random-window read rate a lookup's first windows can reach on this
 * GPU, the practical ceiling of Find beside the HBM copy peak. */
int b2co_oa_window_gather(const b2co_oa_table* table, uint64_t n, uint32_t seed, b2co_stream stream);
/* reference: static_map.h:97 SetErasedKey (static_map.inl:59-66). */
int b2co_oa_set_erased_key(b2co_oa_table* table, uint64_t erased_key_bits, b2co_stream stream);
/* reference: static_map.h:318 Clear, :331 ClearAsync. */
int b2co_oa_clear(b2co_oa_table* table, b2co_stream stream);
int b2co_oa_clear_async(b2co_oa_table* table, b2co_stream stream);

/* Insert (returns the failed count: empty keys, duplicates, full table).
 * reference: static_map.h:116 Insert, static_map.h:131 InsertAsync,
 * open_addressing_impl.h:102-110, kernels.h:46-114. */
int b2co_oa_insert(b2co_oa_table* table, const void* pairs, uint64_t n, b2co_stream stream, uint64_t* failed);
int b2co_oa_insert_async(b2co_oa_table* table, const void* pairs, uint64_t n, b2co_stream stream);
/* InsertIf: only stencil-selected items; failed counts selected items only.
 * reference: static_map.h:216 InsertIf, :237 InsertIfAsync (open_addressing_impl.h:176-218). */
int b2co_oa_insert_if(b2co_oa_table* table, const void* pairs, const uint8_t* stencil, uint64_t n,
                      b2co_stream stream, uint64_t* failed);
int b2co_oa_insert_if_async(b2co_oa_table* table, const void* pairs, const uint8_t* stencil, uint64_t n,
                            b2co_stream stream);
/* InsertOrAssign: failed and assigned (existing keys overwritten) counts.
 * reference: static_map.h:151-175, open_addressing_impl.h:112-156, kernels.h:116-182. */
int b2co_oa_insert_or_assign(b2co_oa_table* table, const void* pairs, uint64_t n, b2co_stream stream,
                             uint64_t* failed, uint64_t* assigned);
int b2co_oa_insert_or_assign_async(b2co_oa_table* table, const void* pairs, uint64_t n, b2co_stream stream);
/* AssignIfAsync: overwrite payloads of existing selected keys, never insert.
 * reference: static_map.h:189, open_addressing_impl.h:158-174, open_addressing_ref_impl.h:384-410. */
int b2co_oa_assign_if_async(b2co_oa_table* table, const void* pairs, const uint8_t* stencil, uint64_t n,
                            b2co_stream stream);
/* InsertAndFind: per input the found payload (T[n]; the key for sets) and a
 * 1-byte inserted flag.  First-wins batches use scratch owned by the table;
 * asynchronous first-wins calls on different streams run on the GPU one after
 * the other, in call order (not while a stream is being captured).
 * reference: static_map.h:256 InsertAndFind, :273 InsertAndFindAsync, open_addressing_impl.h:220-234, kernels.h:212-245. */
int b2co_oa_insert_and_find(b2co_oa_table* table, const void* pairs, void* out_found, uint8_t* out_inserted,
                            uint64_t n, int mode, b2co_stream stream);
int b2co_oa_insert_and_find_async(b2co_oa_table* table, const void* pairs, void* out_found, uint8_t* out_inserted,
                                  uint64_t n, int mode, b2co_stream stream);
/* Sizes the library-owned scratch of first-wins InsertAndFind for batches of
 * up to n items now (4 bytes per item, 4 + 1/4 bytes per slot), so later
 * calls of at most n items allocate nothing and never wait on an allocation.
 * Without it the scratch grows on first use.  No reference counterpart (the
 * reference's InsertAndFind needs no scratch). */
int b2co_oa_reserve_insert_and_find(b2co_oa_table* table, uint64_t n);
/* First-wins InsertAndFind that allocates nothing, for callers that cannot
 * let a library allocate device memory (an application that owns all device
 * memory through its own arena under a fixed budget, or a latency-critical
 * path that must not pay for a device allocation).  No counterpart in the
 * reference.  Same results as b2co_oa_insert_and_find(..., B2CO_IAF_FIRST_WINS)
 * and synchronous like it, but the scratch (4 bytes per item, 4 + 1/4 bytes
 * per table slot) comes from a fixed 32 MiB device array inside the library,
 * which every GPU that loads the library holds until the process exits.
 * Batches needing more scratch fail with B2CO_ERANGE.  Every call looks up
 * the array's address on the current device.  The call ends by synchronizing
 * its stream, so it cannot be captured into a CUDA graph.  All calls share the
 * array, so calls that overlap on the GPU race: serialize them. */
int b2co_oa_insert_and_find_noalloc(b2co_oa_table* table, const void* pairs, void* out_found, uint8_t* out_inserted,
                                    uint64_t n, b2co_stream stream);
/* Erase (returns the count of keys not erased).
 * reference: static_map.h:292 Erase, :307 EraseAsync, open_addressing_impl.h:236-276, open_addressing_ref_impl.h:340-379. */
int b2co_oa_erase(b2co_oa_table* table, const void* keys, uint64_t n, b2co_stream stream, uint64_t* failed);
int b2co_oa_erase_async(b2co_oa_table* table, const void* keys, uint64_t n, b2co_stream stream);
/* Find / FindIf: out[i] = payload of keys[i] or the empty payload.
 * reference: static_map.h:350 Find, :369 FindAsync, :395 FindIf, :419 FindIfAsync, open_addressing_impl.h:278-299, kernels.h:313-347. */
int b2co_oa_find(b2co_oa_table* table, const void* keys, void* out, uint64_t n, b2co_stream stream);
int b2co_oa_find_async(b2co_oa_table* table, const void* keys, void* out, uint64_t n, b2co_stream stream);
int b2co_oa_find_if(b2co_oa_table* table, const void* keys, const uint8_t* stencil, void* out, uint64_t n,
                    b2co_stream stream);
int b2co_oa_find_if_async(b2co_oa_table* table, const void* keys, const uint8_t* stencil, void* out, uint64_t n,
                          b2co_stream stream);
/* Contains / ContainsIf: 1-byte bool per key.
 * reference: static_map.h:439 Contains, :459 ContainsAsync, :485 ContainsIf, :509 ContainsIfAsync, open_addressing_impl.h:301-322, kernels.h:349-377. */
int b2co_oa_contains(b2co_oa_table* table, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
int b2co_oa_contains_async(b2co_oa_table* table, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
int b2co_oa_contains_if(b2co_oa_table* table, const void* keys, const uint8_t* stencil, uint8_t* out, uint64_t n,
                        b2co_stream stream);
int b2co_oa_contains_if_async(b2co_oa_table* table, const void* keys, const uint8_t* stencil, uint8_t* out,
                              uint64_t n, b2co_stream stream);
/* Count: number of keys contained.
 * reference: static_map.h:575, open_addressing_impl.h:446-474, kernels.h:427-467. */
int b2co_oa_count(b2co_oa_table* table, const void* keys, uint64_t n, b2co_stream stream, uint64_t* count);
/* Find with HOST key and output buffers: the batch is split into chunks whose
 * copies in and out overlap the probing on two extra streams.  Same results
 * as b2co_oa_find; the end-to-end form of the reference's Find for callers
 * whose data lives in host memory.
 * reference: static_map.h:350 Find (host staging is the caller's job there). */
int b2co_oa_find_host(b2co_oa_table* table, const void* host_keys, void* host_out, uint64_t n,
                      b2co_stream stream);

/* Kernel shape used by Find/Contains on this table: lanes per key (1, 2, 4 or
 * 8) and keys in flight per lane group (1, 2 or 4), optionally OR-ed with
 * B2CO_FIND_SEGMENTED (scan each first bucket window by 64-byte segments and
 * read the second segment only when the first does not end the scan) and the
 * flags below; 0, 0 = library default (4 lanes, 2 windows, B2CO_FIND_DEFERRED;
 * 2 lanes, 1 window for 4-byte slots and for tables of at most 320 MiB, which
 * are served mostly from L2).  No reference counterpart (the reference
 * launches one thread per key). */
#define B2CO_FIND_SEGMENTED 0x100u
/* OR-ed into keys_per_lane: fetch every first bucket window with one bulk (TMA)
 * copy into shared memory; tables with 16-byte slots only (others ignore it). */
#define B2CO_FIND_BULK 0x200u
/* OR-ed into keys_per_lane: every warp stages its own key chunks (no block barrier). */
#define B2CO_FIND_WARP_STAGED 0x400u
/* OR-ed into keys_per_lane: warp-staged keys, and keys whose first bucket window
 * does not settle them are queued and followed a whole pass at a time. */
#define B2CO_FIND_DEFERRED 0x800u
int b2co_oa_set_find_shape(b2co_oa_table* table, uint32_t lanes_per_key, uint32_t keys_per_lane);
/* Kernel shape of the insert family (Insert, InsertIf, InsertOrAssign,
 * InsertAndFind) for this table (no reference counterpart; results do not
 * depend on it).  lanes_per_key 1 runs one lane per key (the reference's scan
 * as written); 2, 4 or 8 lanes share each bucket window with keys_per_tile
 * (1, 2 or 4) keys in flight per lane group.  (0, 0) restores the default:
 * 4 lanes, 1 key (one lane per key for bucket size 1 and for tables of at
 * most 320 MiB, whose windows mostly come from L2).  Layouts with 2-byte
 * or floating-point keys run the default window shape for any request other
 * than one lane per key. */
int b2co_oa_set_write_shape(b2co_oa_table* table, uint32_t lanes_per_key, uint32_t keys_per_tile);

/* ===================================================================== */
/* Table groups: many independent tables, one launch per operation          */
/* ===================================================================== */
/* The batched pattern (thousands of StaticMap/StaticSet tables of uneven
 * sizes, e.g. per-partition group-by or join builds).  Each table keeps the
 * single-table semantics of b2co_oa_*; the group packs them into one slab and
 * serves an operation on all tables with one persistent launch.  Items of
 * table t are [offsets[t], offsets[t+1]) of a concatenated input (count + 1
 * offsets).  No reference counterpart: the reference runs one launch per
 * container call. */
typedef struct b2co_oa_group b2co_oa_group;

int b2co_oa_group_create(const b2co_oa_desc* desc, const uint64_t* requested_capacities, uint32_t count,
                         b2co_stream stream, b2co_oa_group** out);
int b2co_oa_group_destroy(b2co_oa_group* group);
int b2co_oa_group_table_capacity(const b2co_oa_group* group, uint32_t table, uint64_t* capacity);
int b2co_oa_group_total_slots(const b2co_oa_group* group, uint64_t* slots);
/* The slab: table t's slots start at the sum of the capacities of tables < t. */
int b2co_oa_group_data(const b2co_oa_group* group, void** slab);
int b2co_oa_group_clear(b2co_oa_group* group, b2co_stream stream);
/* Insert into every table (device offsets); with `failed` non-NULL the call
 * synchronizes and returns the total failed count. */
int b2co_oa_group_insert(b2co_oa_group* group, const void* pairs, const uint64_t* d_offsets, uint64_t n,
                         b2co_stream stream, uint64_t* failed);
/* Find (contains = 0) or Contains (contains = 1) on every table, one launch. */
int b2co_oa_group_find(b2co_oa_group* group, const void* keys, const uint64_t* d_offsets, void* out, uint64_t n,
                       int contains, b2co_stream stream);
/* The same launch replayed from a CUDA graph captured on first use. */
int b2co_oa_group_find_graph(b2co_oa_group* group, const void* keys, const uint64_t* d_offsets, void* out,
                             uint64_t n, int contains, b2co_stream stream);
/* One plain launch per table (host offsets): the baseline the group launch replaces. */
int b2co_oa_group_find_per_table(b2co_oa_group* group, const void* keys, const uint64_t* h_offsets, void* out,
                                 int contains, b2co_stream stream);
int b2co_oa_group_insert_per_table(b2co_oa_group* group, const void* pairs, const uint64_t* h_offsets,
                                   b2co_stream stream);
/* Kernel shape of the group Find: lanes per bucket window (1, 2, 4 or 8),
 * keys in flight per lane group (1, 2 or 4, at most the lanes; above 1 the
 * keys whose first window settles nothing are queued and followed a pass at a
 * time) and threads per block (64, 128 or 256; 0 = 256).  Results do not
 * depend on it.  The default is 4 lanes, 2 keys, 256 threads.  The lanes-only
 * form sets one key per lane group. */
int b2co_oa_group_set_find_shape(b2co_oa_group* group, uint32_t lanes);
int b2co_oa_group_set_find_shape_ex(b2co_oa_group* group, uint32_t lanes, uint32_t keys_per_tile, uint32_t block);
int b2co_oa_group_get_find_shape(const b2co_oa_group* group, uint32_t* lanes, uint32_t* keys_per_tile,
                                 uint32_t* block);
/* Autotuner: times every group Find shape (lanes x keys per lane group x
 * threads per block) on this batch, keeps the fastest, and leaves valid
 * results in `out`.  The choice is cached under (operation, key bytes,
 * payload bytes, bucket size, log2 of the mean table capacity) and a later
 * call with the same key reuses it without timing (*from_cache = 1).  The
 * cache lives in the process; b2co_tune_cache_save / _load write and read it
 * as a text file, and a file named by the B2CO_TUNE_CACHE environment
 * variable is loaded on first use and rewritten after every new result.  The
 * lanes-only form reports the lanes of the chosen shape.  No reference
 * counterpart (the batched pattern is this library's). */
int b2co_oa_group_autotune(b2co_oa_group* group, const void* keys, const uint64_t* d_offsets, void* out, uint64_t n,
                           b2co_stream stream, uint32_t* lanes, uint32_t* keys_per_tile, uint32_t* block,
                           int* from_cache);
int b2co_oa_group_autotune_find(b2co_oa_group* group, const void* keys, const uint64_t* d_offsets, void* out,
                                uint64_t n, b2co_stream stream, uint32_t* chosen_lanes);
int b2co_tune_cache_save(const char* path);
int b2co_tune_cache_load(const char* path);
int b2co_tune_cache_clear(void);

/* ===================================================================== */
/* Request server over resident tables                                      */
/* ===================================================================== */
/* The serving pattern: requests of uneven sizes against resident tables,
 * admitted as launch slots and an HBM budget free up, with the arrived
 * Find/Contains requests on one table coalesced into one launch (never past a
 * write on that table: each request sees exactly the writes that arrived
 * before it), and work of many requests overlapping on the device.  A request
 * carries its arrival time (b2co_server_now_ns() clock; 0 = now), so a whole
 * arrival schedule can be submitted ahead of time; requests must be submitted
 * in arrival order.  Host buffers should be pinned.  No reference
 * counterpart. */
typedef enum { B2CO_OP_FIND = 0, B2CO_OP_CONTAINS = 1, B2CO_OP_INSERT = 2, B2CO_OP_INSERT_OR_ASSIGN = 3 } b2co_op;
typedef struct {
    uint64_t id;
    int32_t op;
    int32_t status;       /* b2co_status of the request */
    uint64_t n;
    uint64_t arrival_ns;  /* b2co_server_now_ns() clock */
    uint64_t admit_ns;
    uint64_t done_ns;     /* when the dispatcher saw the launch complete */
    uint64_t failed;      /* Insert / InsertOrAssign counts */
    uint64_t assigned;
} b2co_request_info;
typedef struct b2co_server b2co_server;

uint64_t b2co_server_now_ns(void);
/* max_inflight launch slots (streams); staging plus registered tables never
 * exceed hbm_budget_bytes; coalesced lookups hold at most max_batch_keys keys
 * (0 = 16 Mi).  Every slot's staging buffer is allocated here, sized for a full
 * coalesced lookup batch (at most a quarter of the budget in all). */
int b2co_server_create(uint32_t max_inflight, uint64_t hbm_budget_bytes, uint64_t max_batch_keys, b2co_server** out);
/* Counts a resident table's bytes against the budget. */
int b2co_server_register_table(b2co_server* server, b2co_oa_table* table);
/* Plain mode (non-zero), the baseline the server is measured against: no
 * coalescing, every request its own copy in, launch and copy out, and at most
 * one request per table on the GPU at a time (a table's next request waits
 * for the previous one to finish; different tables still overlap).  Set it
 * while no request is queued. */
int b2co_server_set_plain(b2co_server* server, int plain);
/* Packed copies (off by default): the requests of a coalesced launch are packed
 * by a small pool of host threads into a pinned arena of the launch slot, so
 * the launch issues one host-to-device and one device-to-host copy instead of
 * one per request each way; results are scattered back to each request's
 * buffer before it completes.  The copy engines' rate of operations, not
 * their bandwidth, limits a server of many small requests; with mid-sized
 * requests the host copies cost more than the copy operations they save.
 * The arenas (24 bytes per key of a launch of up to 4 Mi keys, per slot) are
 * allocated with the server; larger launches copy per request. */
int b2co_server_set_packing(b2co_server* server, int on);
/* Direct results (off by default): a lookup launch whose requests' result
 * buffers are pinned host memory gets its results written into them by the
 * GPU (one small kernel of SM stores over PCIe per launch) instead of one
 * device-to-host copy per request, so a lookup costs the copy engines one
 * operation, its keys in.  Requests with pageable result buffers are copied
 * as before.  In plain mode the same applies per request.  Measured on the
 * served benchmark it moves the same bytes over the same bus, so throughput
 * is unchanged; it is off by default because its extra kernel per launch
 * raised p99 latency at moderate rates. */
int b2co_server_set_direct_results(b2co_server* server, int on);
/* host_in: keys (Find/Contains) or pairs (Insert/InsertOrAssign); host_out:
 * payloads (Find) or 1-byte flags (Contains), unused otherwise. */
int b2co_server_submit(b2co_server* server, b2co_oa_table* table, int op, const void* host_in, void* host_out,
                       uint64_t n, uint64_t arrival_ns, uint64_t* request_id);
/* Blocks until the request completes; fills *info and releases the id. */
int b2co_server_wait(b2co_server* server, uint64_t request_id, b2co_request_info* info);
/* One request of a batched submission (the arguments of b2co_server_submit). */
typedef struct {
    b2co_oa_table* table;
    int32_t op;
    int32_t reserved;  /* 0 */
    const void* host_in;
    void* host_out;
    uint64_t n;
    uint64_t arrival_ns;
} b2co_request_desc;
/* Submits `count` requests under one lock, all or none (the first invalid one
 * fails the call); ids[i] is requests[i]'s id. */
int b2co_server_submit_many(b2co_server* server, uint64_t count, const b2co_request_desc* requests, uint64_t* ids);
/* Waits for every id; infos may be NULL.  Returns B2CO_OK, or the status of
 * the first request that failed (all ids are released either way). */
int b2co_server_wait_many(b2co_server* server, uint64_t count, const uint64_t* ids, b2co_request_info* infos);
int b2co_server_stats(b2co_server* server, uint64_t* launches, uint64_t* requests_launched, uint64_t* bytes_in_use);
/* Dispatcher observability, cumulative since creation. */
typedef struct {
    uint64_t launches;
    uint64_t requests_launched;
    uint64_t bytes_in_use;          /* registered tables + staging buffers */
    uint64_t staging_bytes;         /* staging buffers held by the launch slots */
    uint64_t staging_grows;         /* staging (re)allocations */
    uint64_t max_launch_host_ns;    /* longest host time issuing one launch (copies, kernel, event) */
    uint64_t max_reserve_host_ns;   /* longest host time growing a staging buffer */
    uint64_t max_loop_gap_ns;       /* longest interval between two dispatcher polls */
    uint64_t total_launch_host_ns;  /* host time issuing all launches */
    uint64_t copies;                /* host<->device copies issued */
    uint64_t packed_launches;       /* coalesced launches whose requests shared one copy each way */
    uint64_t direct_launches;       /* lookup launches whose results the GPU wrote into the host buffers */
} b2co_server_stats_ex;
int b2co_server_get_stats_ex(b2co_server* server, b2co_server_stats_ex* stats);
/* Finishes every submitted request, then stops the dispatcher. */
int b2co_server_destroy(b2co_server* server);

/* ===================================================================== */
/* StaticMultiset<Key> / StaticMultimap<Key, Value>, Key and Value int32 or  */
/* int64                                                                   */
/* ===================================================================== */
/* The reference's containers expose no slot layout (no Data()); results are
 * defined by the stored entries and the reference's ordering rules, which
 * these follow.  Capacities are exact element counts up to 2^31.  All calls
 * are synchronous, like the reference's (include/static_multiset.h,
 * include/static_multimap.h).  Stencils are uint8 (nonzero = selected). */
typedef struct b2co_mset b2co_mset;
/* reference: static_multiset.h:55 (capacity 0 -> EINVAL). */
int b2co_mset_create(uint64_t capacity, uint32_t key_bytes, uint64_t empty_key_bits, b2co_stream stream,
                     b2co_mset** out);
int b2co_mset_destroy(b2co_mset* set);
int b2co_mset_capacity(const b2co_mset* set, uint64_t* capacity);
int b2co_mset_size(const b2co_mset* set, uint64_t* size);
int b2co_mset_clear(b2co_mset* set, b2co_stream stream);
/* reference: static_multiset.h:159-190 Insert / InsertIf: the earliest valid
 * selected keys up to the remaining capacity are kept in input order;
 * *failed = sentinel keys + selected keys beyond the capacity; a NULL key
 * array with n > 0 reports n failed and changes nothing. */
int b2co_mset_insert(b2co_mset* set, const void* keys, uint64_t n, b2co_stream stream, uint64_t* failed);
int b2co_mset_insert_if(b2co_mset* set, const void* keys, const uint8_t* stencil, uint64_t n, b2co_stream stream,
                        uint64_t* failed);
/* reference: static_multiset.h:192-240 Contains(If) (u8), Find(If) (the key
 * or the empty key), :242-260 CountEach / CountEachOuter (uint64, 0 -> 1). */
int b2co_mset_contains(b2co_mset* set, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
int b2co_mset_contains_if(b2co_mset* set, const void* keys, const uint8_t* stencil, uint8_t* out, uint64_t n,
                          b2co_stream stream);
int b2co_mset_find(b2co_mset* set, const void* keys, void* out, uint64_t n, b2co_stream stream);
int b2co_mset_find_if(b2co_mset* set, const void* keys, const uint8_t* stencil, void* out, uint64_t n,
                      b2co_stream stream);
int b2co_mset_count_each(b2co_mset* set, const void* keys, uint64_t* out, uint64_t n, b2co_stream stream);
int b2co_mset_count_each_outer(b2co_mset* set, const void* keys, uint64_t* out, uint64_t n, b2co_stream stream);
/* reference: :290-294 Count (n * Size() not representable -> EOVERFLOW). */
int b2co_mset_count(b2co_mset* set, const void* keys, uint64_t n, b2co_stream stream, uint64_t* total);
/* reference: :296-321 Retrieve: per query in order, `count` (query, stored
 * key) pairs; total > out_capacity -> ERANGE with nothing written. */
int b2co_mset_retrieve(b2co_mset* set, const void* keys, uint64_t n, void* probe_out, void* match_out,
                       uint64_t out_capacity, b2co_stream stream, uint64_t* written);
/* reference: :322-343 RetrieveAll: every stored key in accepted insertion order. */
int b2co_mset_retrieve_all(b2co_mset* set, void* out, uint64_t out_capacity, b2co_stream stream, uint64_t* written);

typedef struct b2co_mmap b2co_mmap;
/* reference: static_multimap.h:402-410 (capacity 0 -> EINVAL). */
int b2co_mmap_create(uint64_t capacity, uint32_t key_bytes, uint32_t value_bytes, uint64_t empty_key_bits,
                     uint64_t empty_value_bits, b2co_stream stream, b2co_mmap** out);
int b2co_mmap_destroy(b2co_mmap* map);
int b2co_mmap_capacity(const b2co_mmap* map, uint64_t* capacity);
int b2co_mmap_size(const b2co_mmap* map, uint64_t* size);
int b2co_mmap_clear(b2co_mmap* map, b2co_stream stream);
/* reference: static_multimap.h:430-460, :288-399 Insert / InsertIf over
 * Pair<Key, Value>: every selected pair is validated first (a sentinel key or
 * value -> EINVAL, nothing inserted); the earliest selected pairs up to the
 * remaining capacity are kept, duplicates included; *failed = selected pairs
 * not admitted. */
int b2co_mmap_insert(b2co_mmap* map, const void* pairs, uint64_t n, b2co_stream stream, uint64_t* failed);
int b2co_mmap_insert_if(b2co_mmap* map, const void* pairs, const uint8_t* stencil, uint64_t n, b2co_stream stream,
                        uint64_t* failed);
/* reference: :461-480 Contains(If) (u8), Find(If) (the smallest value stored
 * under the key, else the empty value; static_multimap_ref.h QueryImpl). */
int b2co_mmap_contains(b2co_mmap* map, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
int b2co_mmap_contains_if(b2co_mmap* map, const void* keys, const uint8_t* stencil, uint8_t* out, uint64_t n,
                          b2co_stream stream);
int b2co_mmap_find(b2co_mmap* map, const void* keys, void* out, uint64_t n, b2co_stream stream);
int b2co_mmap_find_if(b2co_mmap* map, const void* keys, const uint8_t* stencil, void* out, uint64_t n,
                      b2co_stream stream);
/* reference: :481-492 Count (EOVERFLOW as for the multiset). */
int b2co_mmap_count(b2co_mmap* map, const void* keys, uint64_t n, b2co_stream stream, uint64_t* total);
/* reference: :493-510 Retrieve: per query in order, its values ascending;
 * total > out_capacity -> ERANGE with nothing written. */
int b2co_mmap_retrieve(b2co_mmap* map, const void* keys, uint64_t n, void* key_out, void* value_out,
                       uint64_t out_capacity, b2co_stream stream, uint64_t* written);
/* reference: :512-553 RetrieveAll: all pairs, in accepted insertion order. */
int b2co_mmap_retrieve_all(b2co_mmap* map, void* key_out, void* value_out, uint64_t out_capacity,
                           b2co_stream stream, uint64_t* written);

/* ===================================================================== */
/* RoaringBitmap<Key>, Key uint32 or uint64, portable serialization         */
/* ===================================================================== */
typedef struct b2co_roaring b2co_roaring;
/* reference: include/roaring_bitmap.h:49-77 constructors, parse rules of
 * detail/roaring_bitmap/format.h:164-318: the serialized bitmap (cookie
 * 12346 / 12347 32-bit form, or the 64-bit bucketed form for key_bytes 8) is
 * parsed and validated on the host, then copied to the device.
 * available_bytes bounds the parse (UINT64_MAX: the input is trusted, as in
 * the reference's unbounded constructor); malformed or truncated input ->
 * EINVAL, as the reference's std::invalid_argument. */
int b2co_roaring_create(const void* host_bytes, uint64_t available_bytes, uint32_t key_bytes, b2co_stream stream,
                        b2co_roaring** out);
int b2co_roaring_destroy(b2co_roaring* bitmap);
/* Host only: the validation and measurement the constructor runs. */
int b2co_roaring_parse(const void* host_bytes, uint64_t available_bytes, uint32_t key_bytes, uint64_t* num_keys,
                       uint64_t* size_bytes);
/* reference: roaring_bitmap.h:88-108 Contains / ContainsAsync: out[i] (1 byte)
 * = keys[i] is in the bitmap; NULL buffers only with n == 0. */
int b2co_roaring_contains(b2co_roaring* bitmap, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
int b2co_roaring_contains_async(b2co_roaring* bitmap, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
/* reference: roaring_bitmap.h:110-118 Size (keys), SizeBytes, Data (device copy
 * of the serialized bytes); Empty() is Size() == 0. */
int b2co_roaring_size(const b2co_roaring* bitmap, uint64_t* num_keys);
int b2co_roaring_size_bytes(const b2co_roaring* bitmap, uint64_t* size_bytes);
int b2co_roaring_data(const b2co_roaring* bitmap, const uint8_t** device_bytes);

/* ===================================================================== */
/* BloomFilter<Key>, default policy (8 x uint32 words per block, xxh64)     */
/* ===================================================================== */

typedef struct b2co_bloom b2co_bloom;

/* reference: include/bloom_filter.h:59-62, bloom_filter_lifecycle.inl:15-52
 * (numBlocks 0 -> EINVAL, > UINT32_MAX -> ERANGE). */
int b2co_bloom_create(uint64_t num_blocks, uint32_t key_bytes, uint64_t seed, b2co_stream stream, b2co_bloom** out);
/* Any BloomFilterPolicy<Key, xxhash_64<Key>, uint32_t, WordsPerBlock, PatternBits, ...>
 * (bloom_filter_policy.h:42-181): blocks of words_per_block uint32 words
 * (a power of two <= 32), pattern_bits bits per key spread evenly over the
 * words (a multiple of words_per_block, <= min(64, 32 * words_per_block));
 * other values -> EINVAL, where the reference fails to compile.  The layout
 * and ConditionalAdd / EarlyExitContains parameters change how the reference
 * distributes work, not the bits, so they have no counterpart here.
 * b2co_bloom_create is (8, 8), which is also ArrowFilterPolicy (:211). */
int b2co_bloom_create_policy(uint64_t num_blocks, uint32_t key_bytes, uint64_t seed, uint32_t words_per_block,
                             uint32_t pattern_bits, b2co_stream stream, b2co_bloom** out);
int b2co_bloom_policy(const b2co_bloom* filter, uint32_t* words_per_block, uint32_t* pattern_bits);
int b2co_bloom_destroy(b2co_bloom* filter);
int b2co_bloom_data(const b2co_bloom* filter, uint32_t** words);
int b2co_bloom_num_blocks(const b2co_bloom* filter, uint64_t* num_blocks);
/* reference: bloom_filter.h:66-67 Clear / ClearAsync. */
int b2co_bloom_clear(b2co_bloom* filter, b2co_stream stream);
int b2co_bloom_clear_async(b2co_bloom* filter, b2co_stream stream);
/* reference: bloom_filter.h:69-72 Add / AddAsync / AddIf / AddIfAsync
 * (bloom_filter_impl.h:40-47, bloom_filter_add.inl:15-89). */
int b2co_bloom_add(b2co_bloom* filter, const void* keys, uint64_t n, b2co_stream stream);
/* How Add of the default policy (8 words per block, one bit per word) updates
 * the filter; the bits set are the same either way.  B2CO_BLOOM_ADD_ATOMIC:
 * four 64-bit atomic ORs per key from the SM.  B2CO_BLOOM_ADD_BULK: one
 * 32-byte TMA bulk reduction (OR) per key from shared memory.
 * B2CO_BLOOM_ADD_PARTITIONED: keys are routed by 128 KiB filter slice into a
 * record workspace (8 bytes per key, at most 2^27 keys per round, allocated on
 * first use and kept with the filter), then each slice is built in shared
 * memory and ORed into the filter; filters above 2048 slices (256 MiB) use BULK.
 * B2CO_BLOOM_ADD_AUTO (the default): PARTITIONED for filters of at least 64 MiB
 * and batches of at least 8 keys per filter block, BULK otherwise -- the
 * reference likewise chooses between
 * atomics and a routed path by batch size (bloom_filter_launch.inl:131-240). */
typedef enum {
    B2CO_BLOOM_ADD_ATOMIC = 0,
    B2CO_BLOOM_ADD_BULK = 1,
    B2CO_BLOOM_ADD_PARTITIONED = 2,
    B2CO_BLOOM_ADD_AUTO = 3
} b2co_bloom_add_mode;
int b2co_bloom_set_add_mode(b2co_bloom* filter, int mode);
/* Asynchronous partitioned Adds on different streams share the filter's
 * workspace and run on the GPU one after the other, in call order (not while
 * a stream is being captured); the other Add modes need no ordering. */
int b2co_bloom_add_async(b2co_bloom* filter, const void* keys, uint64_t n, b2co_stream stream);
int b2co_bloom_add_if(b2co_bloom* filter, const void* keys, const uint8_t* stencil, uint64_t n, b2co_stream stream);
int b2co_bloom_add_if_async(b2co_bloom* filter, const void* keys, const uint8_t* stencil, uint64_t n,
                            b2co_stream stream);
/* reference: bloom_filter.h:74-81 Contains / ContainsAsync / ContainsIf
 * (bloom_filter_query.inl:15-120, bloom_filter_impl.h:49-56). */
int b2co_bloom_contains(b2co_bloom* filter, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
int b2co_bloom_contains_async(b2co_bloom* filter, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
int b2co_bloom_contains_if(b2co_bloom* filter, const void* keys, const uint8_t* stencil, uint8_t* out, uint64_t n,
                           b2co_stream stream);
int b2co_bloom_contains_if_async(b2co_bloom* filter, const void* keys, const uint8_t* stencil, uint8_t* out,
                                 uint64_t n, b2co_stream stream);
/* reference: bloom_filter.h:83-87 Merge / MergeAsync / Intersect / IntersectAsync
 * (bloom_filter_merge.inl:15-69; incompatible filters -> EINVAL, bloom_filter_query.inl:197-215). */
int b2co_bloom_merge(b2co_bloom* filter, const b2co_bloom* other, b2co_stream stream);
int b2co_bloom_merge_async(b2co_bloom* filter, const b2co_bloom* other, b2co_stream stream);
int b2co_bloom_intersect(b2co_bloom* filter, const b2co_bloom* other, b2co_stream stream);
int b2co_bloom_intersect_async(b2co_bloom* filter, const b2co_bloom* other, b2co_stream stream);

/* ===================================================================== */
/* HyperLogLog<Key> (int32 / int64 keys, precision 13..18)                 */
/* ===================================================================== */

typedef struct b2co_hll b2co_hll;

/* reference: include/hyperloglog.h:28-30, hyperloglog.inl:115-141
 * (CreateWithSketchSizeKB / CreateWithPrecision / CreateWithStandardDeviation). */
int b2co_hll_precision_for_sketch_kb(uint32_t sketch_kb, uint32_t* precision);
int b2co_hll_precision_for_deviation(double deviation, uint32_t* precision);
int b2co_hll_create(uint32_t precision, uint32_t key_bytes, b2co_stream stream, b2co_hll** out);
int b2co_hll_destroy(b2co_hll* sketch);
/* Registers: 2^precision bytes, register i at byte i.  reference: hyperloglog.h:42 Data(). */
int b2co_hll_data(const b2co_hll* sketch, const uint8_t** registers);
int b2co_hll_precision(const b2co_hll* sketch, uint32_t* precision);
/* reference: hyperloglog.h:37-40 Clear / Add / Merge / Estimate
 * (hyperloglog.inl:215-345). */
int b2co_hll_clear(b2co_hll* sketch, b2co_stream stream);
int b2co_hll_add(b2co_hll* sketch, const void* keys, uint64_t n, b2co_stream stream);
int b2co_hll_add_async(b2co_hll* sketch, const void* keys, uint64_t n, b2co_stream stream);
int b2co_hll_merge(b2co_hll* sketch, const b2co_hll* other, b2co_stream stream);
int b2co_hll_estimate(const b2co_hll* sketch, b2co_stream stream, uint64_t* estimate);
/* The 65-bin rank histogram Estimate reduces (hyperloglog.inl:327-338). */
int b2co_hll_histogram(const b2co_hll* sketch, b2co_stream stream, uint32_t* host_hist65);
/* HLL++ finalizer on a histogram (detail/hyperloglog/finalizer.h:46-74). */
int b2co_hll_finalize(uint32_t precision, const uint32_t* hist65, uint64_t* estimate);
/* The finalizer's interpolation data for a precision (read-only views). */
int b2co_hll_bias_data(uint32_t precision, const double** raw_estimates, const double** biases, uint32_t* points,
                       double* threshold);

/* ===================================================================== */
/* DynamicMap<K,T>: growing set of StaticMap submaps                        */
/* ===================================================================== */

typedef struct b2co_dmap b2co_dmap;

/* reference: include/dynamic_map.h:94-133 (emptyKey == erasedKey -> EINVAL).
 * Key types and slot layouts as for StaticMap (the submaps check them). */
int b2co_dmap_create(const b2co_oa_desc* desc, uint64_t initial_capacity, b2co_stream stream, b2co_dmap** out);
int b2co_dmap_destroy(b2co_dmap* map);
/* reference: dynamic_map.h:137-139 Size / Capacity / NumSubmaps. */
int b2co_dmap_size(const b2co_dmap* map, uint64_t* size);
int b2co_dmap_capacity(const b2co_dmap* map, uint64_t* capacity);
int b2co_dmap_num_submaps(const b2co_dmap* map, uint64_t* count);
/* reference: dynamic_map.h:142-166 Reserve. */
int b2co_dmap_reserve(b2co_dmap* map, uint64_t n, b2co_stream stream);
/* Insert returns the number inserted; mode 0 = kExactDedup, 1 = kAppendUnique.
 * reference: dynamic_map.h:168-219. */
int b2co_dmap_insert(b2co_dmap* map, const void* pairs, uint64_t n, int mode, b2co_stream stream,
                     uint64_t* inserted);
/* InsertOrAssign returns the number of NEW keys (assignments are not counted).
 * reference: dynamic_map.h:237-260, :549-575. */
int b2co_dmap_insert_or_assign(b2co_dmap* map, const void* pairs, uint64_t n, b2co_stream stream, uint64_t* done);
/* reference: dynamic_map.h:262-316 Find / Contains. */
int b2co_dmap_find(b2co_dmap* map, const void* keys, void* out, uint64_t n, b2co_stream stream);
int b2co_dmap_contains(b2co_dmap* map, const void* keys, uint8_t* out, uint64_t n, b2co_stream stream);
/* reference: dynamic_map.h:318-347 Erase (returns the count erased). */
int b2co_dmap_erase(b2co_dmap* map, const void* keys, uint64_t n, b2co_stream stream, uint64_t* erased);
/* reference: dynamic_map.h:349-357 Clear. */
int b2co_dmap_clear(b2co_dmap* map, b2co_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* B2CO_H */
