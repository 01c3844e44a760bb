/*
 * oracle.c -- sequential CPU restatement of the ops-collections bulk-container
 * algorithms.  TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the
 * CUDA product path and the timed CPU baseline, never part of the product.
 *
 * Reference citations are paths inside the reference project.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* hashes                                                                    */
/* ------------------------------------------------------------------------ */

static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
static inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
static inline uint32_t ld32(const uint8_t* p) { uint32_t v; memcpy(&v, p, 4); return v; }
static inline uint64_t ld64(const uint8_t* p) { uint64_t v; memcpy(&v, p, 8); return v; }

/* XXH32: include/detail/hash_functions/xxhash.h:52-175 (canonical XXH32). */
uint32_t orc_xxh32(const void* data, size_t len, uint32_t seed)
{
    const uint32_t P1 = 0x9e3779b1u, P2 = 0x85ebca77u, P3 = 0xc2b2ae3du, P4 = 0x27d4eb2fu, P5 = 0x165667b1u;
    const uint8_t* b = (const uint8_t*)data;
    size_t off = 0;
    uint32_t h;
    if (len >= 16) {
        uint32_t v1 = seed + P1 + P2, v2 = seed + P2, v3 = seed, v4 = seed - P1;
        do {
            v1 = rotl32(v1 + ld32(b + off) * P2, 13) * P1;
            v2 = rotl32(v2 + ld32(b + off + 4) * P2, 13) * P1;
            v3 = rotl32(v3 + ld32(b + off + 8) * P2, 13) * P1;
            v4 = rotl32(v4 + ld32(b + off + 12) * P2, 13) * P1;
            off += 16;
        } while (off <= len - 16);
        h = rotl32(v1, 1) + rotl32(v2, 7) + rotl32(v3, 12) + rotl32(v4, 18);
    } else {
        h = seed + P5;
    }
    h += (uint32_t)len;
    for (; off + 4 <= len; off += 4) h = rotl32(h + ld32(b + off) * P3, 17) * P4;
    for (; off < len; ++off) h = rotl32(h + (uint32_t)b[off] * P5, 11) * P1;
    h ^= h >> 15; h *= P2; h ^= h >> 13; h *= P3; h ^= h >> 16;
    return h;
}

/* XXH64: include/detail/hash_functions/xxhash.h:184-326 (canonical XXH64;
 * the 4- and 8-byte fast paths at :199-218 equal the generic tail). */
uint64_t orc_xxh64(const void* data, size_t len, uint64_t seed)
{
    const uint64_t P1 = 11400714785074694791ull, P2 = 14029467366897019727ull, P3 = 1609587929392839161ull,
                   P4 = 9650029242287828579ull, P5 = 2870177450012600261ull;
    const uint8_t* b = (const uint8_t*)data;
    size_t off = 0;
    uint64_t h;
    if (len >= 32) {
        uint64_t v[4] = {seed + P1 + P2, seed + P2, seed, seed - P1};
        do {
            for (int i = 0; i < 4; ++i) v[i] = rotl64(v[i] + ld64(b + off + 8 * i) * P2, 31) * P1;
            off += 32;
        } while (off <= len - 32);
        h = rotl64(v[0], 1) + rotl64(v[1], 7) + rotl64(v[2], 12) + rotl64(v[3], 18);
        for (int i = 0; i < 4; ++i) {
            uint64_t k = rotl64(v[i] * P2, 31) * P1;
            h = (h ^ k) * P1 + P4;
        }
    } else {
        h = seed + P5;
    }
    h += (uint64_t)len;
    for (; off + 8 <= len; off += 8) {
        uint64_t k = rotl64(ld64(b + off) * P2, 31) * P1;
        h = rotl64(h ^ k, 27) * P1 + P4;
    }
    for (; off + 4 <= len; off += 4) h = rotl64(h ^ ((uint64_t)ld32(b + off) * P1), 23) * P2 + P3;
    for (; off < len; ++off) h = rotl64(h ^ ((uint64_t)b[off] * P5), 11) * P1;
    h ^= h >> 33; h *= P2; h ^= h >> 29; h *= P3; h ^= h >> 32;
    return h;
}

/* fmix32 / fmix64: include/detail/hash_functions/utils.h:42-66 (key ^ seed, then the
 * MurmurHash3 finalizer). */
uint32_t orc_fmix32(uint32_t k, uint32_t seed)
{
    uint32_t h = k ^ seed;
    h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
    return h;
}
uint64_t orc_fmix64(uint64_t k, uint64_t seed)
{
    uint64_t h = k ^ seed;
    h ^= h >> 33; h *= 0xff51afd7ed558ccdull; h ^= h >> 33; h *= 0xc4ceb9fe1a85ec53ull; h ^= h >> 33;
    return h;
}

/* MurmurHash3_x86_32: include/detail/hash_functions/murmurhash3.h:57-106. */
uint32_t orc_murmur3_32(const void* data, size_t len, uint32_t seed)
{
    const uint8_t* b = (const uint8_t*)data;
    const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    size_t nblocks = len / 4;
    uint32_t h = seed;
    for (size_t i = 0; i < nblocks; ++i) {
        uint32_t k = ld32(b + 4 * i);
        k *= c1; k = rotl32(k, 15); k *= c2;
        h ^= k; h = rotl32(h, 13); h = h * 5 + 0xe6546b64u;
    }
    uint32_t k = 0;
    switch (len & 3) {
        case 3: k ^= (uint32_t)b[nblocks * 4 + 2] << 16; /* fall through */
        case 2: k ^= (uint32_t)b[nblocks * 4 + 1] << 8;  /* fall through */
        case 1: k ^= (uint32_t)b[nblocks * 4]; k *= c1; k = rotl32(k, 15); k *= c2; h ^= k;
    }
    h ^= (uint32_t)len;
    return orc_fmix32(h, 0);
}

/* The probing schemes cast the hash result to the kernels' uint32 size type
 * (utility/math_utils.h:14-24 SanitizeHash; kernels pass uint32 tableSize). */
uint32_t orc_probe_hash(int kind, uint64_t key_bits, uint32_t key_bytes, uint32_t seed)
{
    uint8_t kb[8];
    memcpy(kb, &key_bits, 8);
    switch (kind) {
        case ORC_HASH_XXH32: return orc_xxh32(kb, key_bytes, seed);
        case ORC_HASH_MURMUR3_32: return orc_murmur3_32(kb, key_bytes, seed);
        case ORC_HASH_FMIX:  /* Fmix32/Fmix64 take 4- or 8-byte keys only (utils.h:42-66) */
            return key_bytes == 4 ? orc_fmix32((uint32_t)key_bits, seed) : (uint32_t)orc_fmix64(key_bits, seed);
        case ORC_HASH_XXH64: return (uint32_t)orc_xxh64(kb, key_bytes, seed);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* capacity prime table                                                      */
/* ------------------------------------------------------------------------ */
/* include/utility/prime.h:15 holds 140,741 primes.  They follow a fixed rule,
 * verified entry by entry against that table: 2,3,5,7,11,13; then each next
 * entry is the smallest prime >= previous + 6 (with 151 listed directly after
 * 149) up to 131,101; from there each next entry is the smallest prime >=
 * previous + 2^17.  The oracle regenerates the table from that rule. */

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)((__uint128_t)a * b % m); }
static uint64_t powmod(uint64_t a, uint64_t e, uint64_t m)
{
    uint64_t r = 1;
    a %= m;
    while (e) {
        if (e & 1) r = mulmod(r, a, m);
        a = mulmod(a, a, m);
        e >>= 1;
    }
    return r;
}
static int is_prime_u64(uint64_t n)
{
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; ++i) {
        if (n == small[i]) return 1;
        if (n % small[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; ++s; }
    for (int i = 0; i < 12; ++i) {
        uint64_t x = powmod(small[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int r = 1; r < s; ++r) {
            x = mulmod(x, x, n);
            if (x == n - 1) { comp = 0; break; }
        }
        if (comp) return 0;
    }
    return 1;
}
static uint64_t next_prime(uint64_t n)
{
    while (!is_prime_u64(n)) ++n;
    return n;
}

#define ORC_PRIME_COUNT 140741u
static uint64_t* g_primes;

static void build_primes(void)
{
    if (g_primes) return;
    uint64_t* t = (uint64_t*)malloc(sizeof(uint64_t) * ORC_PRIME_COUNT);
    static const uint64_t head[] = {2, 3, 5, 7, 11, 13};
    uint32_t n = 0;
    for (; n < 6; ++n) t[n] = head[n];
    uint64_t p = 13;
    while (p <= 131072) {
        p = next_prime(p + 6);
        t[n++] = p;
        if (p == 149) { p = 151; t[n++] = p; }
    }
    while (n < ORC_PRIME_COUNT) {
        p = next_prime(p + 131072);
        t[n++] = p;
    }
    g_primes = t;
}

uint64_t orc_prime_table_size(void) { return ORC_PRIME_COUNT; }
uint64_t orc_prime_table_entry(uint64_t i)
{
    build_primes();
    return i < ORC_PRIME_COUNT ? g_primes[i] : 0;
}
uint64_t orc_prime_at_least(uint64_t n)
{
    build_primes();
    /* LowerBound (utility/math_utils.h:74-95) over the sorted table. */
    uint64_t lo = 0, cnt = ORC_PRIME_COUNT;
    while (cnt > 0) {
        uint64_t step = cnt / 2, it = lo + step;
        if (g_primes[it] < n) { lo = it + 1; cnt -= step + 1; } else cnt = step;
    }
    return lo < ORC_PRIME_COUNT ? g_primes[lo] : 0;
}

/* MakeValidExtent: detail/extent/extent.inl:20-41 (double hashing) and :43-60 (linear). */
uint64_t orc_valid_capacity(uint64_t request, uint32_t b, int probing)
{
    uint64_t m = request > 1 ? request : 1;
    uint64_t size = m / b + (m % b != 0);
    if (probing == ORC_PROBE_DOUBLE) {
        uint64_t p = orc_prime_at_least(size);
        return p ? p * b : 0;
    }
    return (size + (request == 0)) * b;
}

/* ------------------------------------------------------------------------ */
/* probing                                                                   */
/* ------------------------------------------------------------------------ */

/* LinearProbing::MakeIterator (probing_scheme_impl.inl:116-128) and
 * DoubleHashing::MakeIterator (:175-189); DoubleHashing's second hash is the
 * same hash family seeded with 1 (probing_scheme.h:99). */
orc_probe_iter orc_make_iter(int probing, int hash_kind, uint64_t key_bits, uint32_t key_bytes, uint32_t b,
                             uint32_t cap)
{
    orc_probe_iter it;
    uint32_t nb = cap / b;
    uint32_t h1 = orc_probe_hash(hash_kind, key_bits, key_bytes, 0);
    it.idx = (h1 % nb) * b;
    if (probing == ORC_PROBE_DOUBLE) {
        uint32_t h2 = orc_probe_hash(hash_kind, key_bits, key_bytes, 1);
        it.step = (h2 % (nb - 1) + 1) * b;
    } else {
        it.step = b;
    }
    it.upper = cap;
    return it;
}

/* ProbingIterator::operator++ (probing_scheme_impl.inl:76-84). */
uint32_t orc_iter_next(orc_probe_iter* it)
{
    uint32_t rem = it->upper - it->step;
    it->idx = it->idx >= rem ? it->idx - rem : it->idx + it->step;
    return it->idx;
}

/* ------------------------------------------------------------------------ */
/* open addressing                                                           */
/* ------------------------------------------------------------------------ */

/* Pair<K,V> is aligned to min(16, bitceil(sizeof K + sizeof V)) (pair.inl:19-24),
 * the payload at the next offset aligned to its own size. */
void orc_slot_layout(uint32_t kb, uint32_t vb, uint32_t* slot_bytes, uint32_t* value_offset)
{
    if (vb == 0) { *slot_bytes = kb; *value_offset = 0; return; }
    uint32_t sum = kb + vb, align = 1;
    while (align < sum) align <<= 1;
    if (align > 16) align = 16;
    uint32_t voff = (kb + vb - 1) / vb * vb;
    uint32_t end = voff + vb;
    *value_offset = voff;
    *slot_bytes = (end + align - 1) / align * align;
}

static inline uint64_t ld_bits(const uint8_t* p, uint32_t n)
{
    uint64_t v = 0;
    memcpy(&v, p, n);
    return v;
}
static inline void st_bits(uint8_t* p, uint64_t v, uint32_t n) { memcpy(p, &v, n); }

static inline uint8_t* slot_ptr(const orc_table* t, uint32_t i) { return t->slots + (size_t)i * t->slot_bytes; }
static inline uint64_t slot_key(const orc_table* t, uint32_t i) { return ld_bits(slot_ptr(t, i), t->key_bytes); }
static inline uint64_t slot_val(const orc_table* t, uint32_t i)
{
    /* A set's "value" is the stored key (open_addressing_ref_impl.h:71-79). */
    return t->value_bytes ? ld_bits(slot_ptr(t, i) + t->value_offset, t->value_bytes) : slot_key(t, i);
}
static inline void write_slot(orc_table* t, uint32_t i, uint64_t k, uint64_t v)
{
    uint8_t* p = slot_ptr(t, i);
    st_bits(p, k, t->key_bytes);
    if (t->value_bytes) st_bits(p + t->value_offset, v, t->value_bytes);
}
static inline uint64_t empty_payload(const orc_table* t) { return t->value_bytes ? t->empty_value : t->empty_key; }

/* IEEE 754 binary16 -> binary32, exact (every half is a float). */
static float half_to_float(uint16_t h)
{
    uint32_t e = (h >> 10) & 31u, m = h & 1023u;
    float v;
    if (e == 0) v = ldexpf((float)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = ldexpf((float)(m | 1024u), (int)e - 25);
    return (h >> 15) ? -v : v;
}

/* KeyEqual (EqualTo, utility/math_utils.h:66-70 via equal_wrapper.h:30-33):
 * integer keys compare bitwise; floating-point keys with ==, so -0 matches +0
 * and NaN matches nothing.  Sentinel tests stay bitwise everywhere. */
static inline int key_eq(const orc_table* t, uint64_t a, uint64_t b)
{
    if (t->key_kind != ORC_KEY_FLOAT) return a == b;
    if (t->key_bytes == 2) return half_to_float((uint16_t)a) == half_to_float((uint16_t)b);
    if (t->key_bytes == 4) {
        uint32_t ua = (uint32_t)a, ub = (uint32_t)b;
        float x, y;
        memcpy(&x, &ua, 4);
        memcpy(&y, &ub, 4);
        return x == y;
    }
    double x, y;
    memcpy(&x, &a, 8);
    memcpy(&y, &b, 8);
    return x == y;
}

/* Storage initialisation: every slot holds Pair{emptyKey, emptyValue}
 * (open_addressing_impl.h:84-93, bucket_storage.inl:52-64). */
void orc_table_clear(orc_table* t)
{
    memset(t->slots, 0, (size_t)t->capacity * t->slot_bytes);
    for (uint32_t i = 0; i < t->capacity; ++i) write_slot(t, i, t->empty_key, t->empty_value);
}

static inline orc_probe_iter iter_for(const orc_table* t, uint64_t key)
{
    return orc_make_iter(t->probing, t->hash_kind, key, t->key_bytes, t->bucket_size, t->capacity);
}

/* InsertVerdict<assign> (open_addressing_ref_impl.h:489-532): slots equal to the
 * empty key are AVAILABLE, equal keys are DUPLICATE (payload overwritten when
 * assigning), a completed cycle or the empty key itself FAILS. */
static int insert_verdict(orc_table* t, uint64_t key, uint64_t val, int assign, uint32_t* where)
{
    if (key == t->empty_key) return ORC_FAILED;
    orc_probe_iter it = iter_for(t, key);
    uint32_t init = it.idx;
    for (;;) {
        for (uint32_t i = 0; i < t->bucket_size; ++i) {
            uint32_t s = it.idx + i;
            uint64_t sk = slot_key(t, s);
            if (sk == t->empty_key) {
                write_slot(t, s, key, val);
                if (where) *where = s;
                return ORC_SUCCESS;
            }
            if (key_eq(t, sk, key)) {
                if (assign && t->value_bytes) st_bits(slot_ptr(t, s) + t->value_offset, val, t->value_bytes);
                if (where) *where = s;
                return ORC_DUPLICATE;
            }
        }
        if (orc_iter_next(&it) == init) return ORC_FAILED;
    }
}

static inline uint64_t in_key(const orc_table* t, const void* keys, uint64_t i)
{
    return ld_bits((const uint8_t*)keys + i * t->key_bytes, t->key_bytes);
}
static inline uint64_t in_val(const orc_table* t, const void* vals, uint64_t i)
{
    if (!t->value_bytes) return 0;
    return ld_bits((const uint8_t*)vals + i * t->value_bytes, t->value_bytes);
}

/* The sequential bulk forms touch the first bucket window of input i + kAhead
 * early (a cache prefetch, no state change), so a large table is not walked at
 * one DRAM latency per key; results are those of the plain in-order loop. */
enum { kAhead = 16 };
static inline void touch_first_window(const orc_table* t, const void* keys, uint64_t i, uint64_t n)
{
    if (i >= n) return;
    orc_probe_iter it = iter_for(t, in_key(t, keys, i));
    const uint8_t* p = slot_ptr(t, it.idx);
    __builtin_prefetch(p, 1, 0);
    __builtin_prefetch(p + (size_t)t->bucket_size * t->slot_bytes - 1, 1, 0);
}

int orc_key_equal(int key_kind, uint32_t key_bytes, uint64_t a, uint64_t b)
{
    orc_table t;
    memset(&t, 0, sizeof t);
    t.key_kind = key_kind;
    t.key_bytes = key_bytes;
    return key_eq(&t, a, b);
}

/* Insert / InsertIf: kernels.h:46-83; returns the failed count (pred-true items only). */
uint64_t orc_insert(orc_table* t, const void* keys, const void* vals, const uint8_t* stencil, uint64_t n)
{
    uint64_t failed = 0;
    for (uint64_t i = 0; i < n; ++i) {
        touch_first_window(t, keys, i + kAhead, n);
        if (stencil && !stencil[i]) continue;
        if (insert_verdict(t, in_key(t, keys, i), in_val(t, vals, i), 0, NULL) != ORC_SUCCESS) ++failed;
    }
    return failed;
}

/* InsertOrAssign: kernels.h:116-156 -- failed in the return value, assigned
 * (existing keys whose payload was overwritten) through *assigned. */
uint64_t orc_insert_or_assign(orc_table* t, const void* keys, const void* vals, uint64_t n, uint64_t* assigned)
{
    uint64_t failed = 0, asg = 0;
    for (uint64_t i = 0; i < n; ++i) {
        touch_first_window(t, keys, i + kAhead, n);
        int r = insert_verdict(t, in_key(t, keys, i), in_val(t, vals, i), 1, NULL);
        if (r == ORC_FAILED) ++failed;
        else if (r == ORC_DUPLICATE) ++asg;
    }
    if (assigned) *assigned = asg;
    return failed;
}

/* Assign (open_addressing_ref_impl.h:384-410) behind AssignIfAsync (kernels.h:184-210). */
void orc_assign_if(orc_table* t, const void* keys, const void* vals, const uint8_t* stencil, uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i) {
        if (stencil && !stencil[i]) continue;
        uint64_t key = in_key(t, keys, i);
        orc_probe_iter it = iter_for(t, key);
        uint32_t init = it.idx;
        int done = 0;
        while (!done) {
            for (uint32_t j = 0; j < t->bucket_size && !done; ++j) {
                uint32_t s = it.idx + j;
                uint64_t sk = slot_key(t, s);
                if (sk == t->empty_key) { done = 1; break; }
                if (key_eq(t, sk, key)) {
                    st_bits(slot_ptr(t, s) + t->value_offset, in_val(t, vals, i), t->value_bytes);
                    done = 1;
                }
            }
            if (!done && orc_iter_next(&it) == init) done = 1;
        }
    }
}

/* InsertAndFind (open_addressing_ref_impl.h:301-330, 543-565), input order =
 * first occurrence wins, which is the golden the reference's own tests use
 * (tests/common/golden.h:104-131). */
void orc_insert_and_find(orc_table* t, const void* keys, const void* vals, uint64_t n, void* out_found,
                         uint8_t* out_inserted)
{
    uint32_t ob = t->value_bytes ? t->value_bytes : t->key_bytes;
    for (uint64_t i = 0; i < n; ++i) {
        touch_first_window(t, keys, i + kAhead, n);
        uint64_t key = in_key(t, keys, i);
        uint32_t where = 0;
        int r = insert_verdict(t, key, in_val(t, vals, i), 0, &where);
        uint64_t found = r == ORC_FAILED ? empty_payload(t) : slot_val(t, where);
        st_bits((uint8_t*)out_found + i * ob, found, ob);
        out_inserted[i] = r == ORC_SUCCESS;
    }
}

/* FindAndContains (open_addressing_ref_impl.h:567-605).  *windows counts the
 * buckets visited (the per-query probe count used by the roofline). */
static int find_one(const orc_table* t, uint64_t key, uint64_t* val, uint32_t* windows)
{
    orc_probe_iter it = iter_for(t, key);
    uint32_t init = it.idx, w = 0;
    for (;;) {
        ++w;
        for (uint32_t i = 0; i < t->bucket_size; ++i) {
            uint32_t s = it.idx + i;
            uint64_t sk = slot_key(t, s);
            if (sk == t->empty_key) { *val = empty_payload(t); *windows = w; return 0; }
            if (key_eq(t, sk, key)) { *val = slot_val(t, s); *windows = w; return 1; }
        }
        if (orc_iter_next(&it) == init) { *val = empty_payload(t); *windows = w; return 0; }
    }
}

/* FindIf (kernels.h:313-347): stencil-false items get the empty payload. */
void orc_find(const orc_table* t, const void* keys, const uint8_t* stencil, uint64_t n, void* out, uint32_t* wins)
{
    uint32_t ob = t->value_bytes ? t->value_bytes : t->key_bytes;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t v = empty_payload(t);
        uint32_t w = 0;
        if (!stencil || stencil[i]) find_one(t, in_key(t, keys, i), &v, &w);
        st_bits((uint8_t*)out + i * ob, v, ob);
        if (wins) wins[i] = w;
    }
}

void orc_find_parallel(const orc_table* t, const void* keys, uint64_t n, void* out, int threads)
{
    uint32_t ob = t->value_bytes ? t->value_bytes : t->key_bytes;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static, 65536)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t v;
        uint32_t w;
        find_one(t, in_key(t, keys, (uint64_t)i), &v, &w);
        st_bits((uint8_t*)out + (uint64_t)i * ob, v, ob);
    }
    (void)threads;
}

void orc_contains_parallel(const orc_table* t, const void* keys, uint64_t n, uint8_t* out, int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static, 65536)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t v;
        uint32_t w;
        out[i] = (uint8_t)find_one(t, in_key(t, keys, (uint64_t)i), &v, &w);
    }
    (void)threads;
}

static inline int slot_occupied(const orc_table* t, uint32_t s)
{
    uint64_t k = slot_key(t, s);
    return k != t->empty_key && (t->erased_key == t->empty_key || k != t->erased_key);
}

/* Slots [lo, hi) of a: occupied count, and keys b misses or holds with another payload. */
static void pairs_match_range(const orc_table* a, const orc_table* b, uint32_t lo, uint32_t hi, uint64_t* occ,
                              uint64_t* bad)
{
    for (uint32_t s = lo; s < hi; ++s) {
        if (!slot_occupied(a, s)) continue;
        ++*occ;
        uint64_t v;
        uint32_t w;
        if (!find_one(b, slot_key(a, s), &v, &w) || v != slot_val(a, s)) ++*bad;
    }
}

static uint64_t count_occupied(const orc_table* t)
{
    uint64_t c = 0;
    for (uint32_t s = 0; s < t->capacity; ++s) c += (uint64_t)slot_occupied(t, s);
    return c;
}

void orc_pairs_match(const orc_table* a, const orc_table* b, uint64_t* occupied_a, uint64_t* occupied_b,
                     uint64_t* mismatches, int threads)
{
    uint64_t occ_a = 0, occ_b = 0, bad = 0;
    int64_t const chunk = 1 << 20, nchunks = ((int64_t)a->capacity + chunk - 1) / chunk;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : occ_a, bad)
#endif
    for (int64_t c = 0; c < nchunks; ++c) {
        uint64_t hi = (uint64_t)(c + 1) * chunk;
        pairs_match_range(a, b, (uint32_t)(c * chunk), (uint32_t)(hi < a->capacity ? hi : a->capacity), &occ_a,
                          &bad);
    }
    int64_t const nb = ((int64_t)b->capacity + chunk - 1) / chunk;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : occ_b)
#endif
    for (int64_t c = 0; c < nb; ++c) {
        uint64_t hi = (uint64_t)(c + 1) * chunk;
        for (uint32_t s = (uint32_t)(c * chunk); s < (uint32_t)(hi < b->capacity ? hi : b->capacity); ++s)
            occ_b += (uint64_t)slot_occupied(b, s);
    }
    *occupied_a = occ_a;
    *occupied_b = occ_b;
    *mismatches = bad;
    (void)threads;
}

uint64_t orc_group_check(uint64_t count, const uint64_t* caps, const uint64_t* slot_off, const uint8_t* slab,
                         const orc_table* shape, const void* keys, const void* values, const uint64_t* ins_off,
                         const void* queries, const uint64_t* q_off, void* out_expected, uint64_t* first_bad,
                         int threads)
{
    uint64_t bad = 0, first = UINT64_MAX;
    uint32_t const ob = shape->value_bytes ? shape->value_bytes : shape->key_bytes;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad)
#endif
    for (int64_t i = 0; i < (int64_t)count; ++i) {
        orc_table o = *shape, d = *shape;
        o.capacity = d.capacity = (uint32_t)caps[i];
        o.slots = (uint8_t*)malloc((size_t)caps[i] * shape->slot_bytes);
        d.slots = (uint8_t*)slab + slot_off[i] * shape->slot_bytes;
        orc_table_clear(&o);
        uint64_t const k0 = ins_off[i], nk = ins_off[i + 1] - k0;
        orc_insert(&o, (const uint8_t*)keys + k0 * shape->key_bytes,
                   values ? (const uint8_t*)values + k0 * shape->value_bytes : NULL, NULL, nk);
        uint64_t occ = 0, mism = 0;
        pairs_match_range(&o, &d, 0, o.capacity, &occ, &mism);
        if (mism || count_occupied(&d) != occ) {
            ++bad;
#ifdef _OPENMP
#pragma omp critical
#endif
            if ((uint64_t)i < first) first = (uint64_t)i;
        }
        uint64_t const q0 = q_off[i];
        for (uint64_t j = q0; j < q_off[i + 1]; ++j) {
            uint64_t v;
            uint32_t w;
            find_one(&o, in_key(&o, queries, j), &v, &w);
            st_bits((uint8_t*)out_expected + j * ob, v, ob);
        }
        free(o.slots);
    }
    if (first_bad) *first_bad = first;
    (void)threads;
    return bad;
}

/* ContainsIf (kernels.h:349-377). */
void orc_contains(const orc_table* t, const void* keys, const uint8_t* stencil, uint64_t n, uint8_t* out,
                  uint32_t* wins)
{
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t v;
        uint32_t w = 0;
        out[i] = (!stencil || stencil[i]) ? (uint8_t)find_one(t, in_key(t, keys, i), &v, &w) : 0;
        if (wins) wins[i] = w;
    }
}

/* Erase with an optional tombstone (open_addressing_ref_impl.h:340-379): the
 * matched slot becomes {erasedKey, emptyValue}; without a tombstone it becomes
 * the empty slot and the scan never stops early at an empty slot.  Returns the
 * number of keys NOT erased (kernels.h:247-279 counts failures). */
uint64_t orc_erase(orc_table* t, const void* keys, uint64_t n)
{
    uint64_t failed = 0;
    int tomb = t->erased_key != t->empty_key;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t key = in_key(t, keys, i);
        orc_probe_iter it = iter_for(t, key);
        uint32_t init = it.idx;
        int done = 0, ok = 0;
        while (!done) {
            for (uint32_t j = 0; j < t->bucket_size && !done; ++j) {
                uint32_t s = it.idx + j;
                uint64_t sk = slot_key(t, s);
                if (sk == t->empty_key) {
                    if (tomb) done = 1;
                    continue;
                }
                if (key_eq(t, sk, key)) {
                    write_slot(t, s, tomb ? t->erased_key : t->empty_key, t->empty_value);
                    ok = 1;
                    done = 1;
                }
            }
            if (!done && orc_iter_next(&it) == init) done = 1;
        }
        if (!ok) ++failed;
    }
    return failed;
}

/* Count (kernels.h:427-467): the number of queries contained. */
uint64_t orc_count(const orc_table* t, const void* keys, uint64_t n)
{
    uint64_t c = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t v;
        uint32_t w;
        c += (uint64_t)find_one(t, in_key(t, keys, i), &v, &w);
    }
    return c;
}

/* ------------------------------------------------------------------------ */
/* Bloom filter                                                              */
/* ------------------------------------------------------------------------ */

/* The policy's 64-entry salt table (bloom_filter_policy.h:170-178).  The first
 * eight are the split-block Bloom filter salts of the Parquet specification and
 * are all the default policy (8 words per block, PatternBits 8) uses; policies
 * with more pattern bits take salt[w * bitsPerWord + b] for bit b of word w. */
static const uint32_t k_salts[64] = {
    0x47b6137bu, 0x44974d91u, 0x8824ad5bu, 0xa2b7289du, 0x705495c7u, 0x2df1424bu, 0x9efc4947u, 0x5c6bfb31u,
    0xb24bcdffu, 0xb6843d6du, 0x6db04543u, 0x3a12efddu, 0xb0ddd463u, 0x8d22f6e7u, 0xb82f1e53u, 0x7db9f86bu,
    0xc7afe639u, 0xfb135cd7u, 0x693256e1u, 0x9466d871u, 0x23d3d02fu, 0x6461d049u, 0x66a91621u, 0xbaa3006fu,
    0x52fb8d99u, 0x3ea88b4fu, 0x0f470cfdu, 0xb1db79a5u, 0x9809fcd1u, 0xbced4445u, 0x2eb7c737u, 0x2cea6803u,
    0x156f1955u, 0x8813c027u, 0xa26819f9u, 0x4c3b57bdu, 0x7df94487u, 0xb975e769u, 0xb8f20cb5u, 0x5c9e2e77u,
    0x5fb1735fu, 0x3a6f759bu, 0x3c090923u, 0xfced424du, 0xa187a6a9u, 0x6f070a41u, 0x2c85233bu, 0x7e62258bu,
    0x2771ef17u, 0x13bbf093u, 0x4ff059e5u, 0xe3ce3d0fu, 0xf1b4789fu, 0x9fbb6173u, 0x6a320cf5u, 0x1be2c481u,
    0x7ba8222bu, 0x6fd619b3u, 0x7b1bbf0du, 0x8b8993adu, 0x448eca95u, 0x82ab09d9u, 0x2ce53909u, 0x4f548685u};

static inline void bloom_locate(const void* keys, uint32_t kb, uint64_t i, uint64_t nblocks, uint64_t seed,
                                uint32_t* block, uint32_t* lower)
{
    uint64_t h = orc_xxh64((const uint8_t*)keys + i * kb, kb, seed);
    /* BlockIndex: multiply-high of the upper 32 hash bits by uint32(numBlocks)
     * (bloom_filter_policy.h:101-107). */
    *block = (uint32_t)(((uint64_t)(uint32_t)(h >> 32) * (uint32_t)nblocks) >> 32);
    *lower = (uint32_t)h;
}

/* Word w's pattern: bitsPerWord bits, bit b at (salt[w*bpw+b] * lower) >> 27
 * for 32-bit words (WordPatternImpl, bloom_filter_policy.h:146-159). */
uint32_t orc_bloom_word_pattern(uint32_t w, uint32_t bpw, uint32_t lower)
{
    uint32_t pat = 0;
    for (uint32_t b = 0; b < bpw; ++b) pat |= 1u << ((k_salts[w * bpw + b] * lower) >> 27);
    return pat;
}

int orc_bloom_policy_valid(uint32_t wpb, uint32_t pattern_bits)
{
    /* the static_asserts of the policy constructor (bloom_filter_policy.h:60-86), 32-bit words */
    if (wpb == 0 || (wpb & (wpb - 1)) != 0 || wpb > 32) return 0;
    if (pattern_bits < wpb || pattern_bits > 64 || pattern_bits > 32 * wpb || pattern_bits % wpb != 0) return 0;
    return 1;
}

void orc_bloom_add_policy(uint32_t* words, uint64_t nblocks, uint32_t wpb, uint32_t pattern_bits, const void* keys,
                          uint32_t kb, uint64_t n, uint64_t seed)
{
    uint32_t const bpw = pattern_bits / wpb;
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t block, lower;
        bloom_locate(keys, kb, i, nblocks, seed, &block, &lower);
        for (uint32_t w = 0; w < wpb; ++w) words[(uint64_t)block * wpb + w] |= orc_bloom_word_pattern(w, bpw, lower);
    }
}

static inline uint8_t bloom_test(const uint32_t* words, uint32_t wpb, uint32_t bpw, uint32_t block, uint32_t lower)
{
    for (uint32_t w = 0; w < wpb; ++w) {
        uint32_t pat = orc_bloom_word_pattern(w, bpw, lower);
        if ((words[(uint64_t)block * wpb + w] & pat) != pat) return 0;
    }
    return 1;
}

void orc_bloom_contains_policy(const uint32_t* words, uint64_t nblocks, uint32_t wpb, uint32_t pattern_bits,
                               const void* keys, uint32_t kb, uint64_t n, uint64_t seed, uint8_t* out, int threads)
{
    uint32_t const bpw = pattern_bits / wpb;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static, 65536) if (threads != 1)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint32_t block, lower;
        bloom_locate(keys, kb, (uint64_t)i, nblocks, seed, &block, &lower);
        out[i] = bloom_test(words, wpb, bpw, block, lower);
    }
    (void)threads;
}

void orc_bloom_add(uint32_t* words, uint64_t nblocks, const void* keys, uint32_t kb, uint64_t n, uint64_t seed)
{
    orc_bloom_add_policy(words, nblocks, 8, 8, keys, kb, n, seed);
}

void orc_bloom_contains(const uint32_t* words, uint64_t nblocks, const void* keys, uint32_t kb, uint64_t n,
                        uint64_t seed, uint8_t* out)
{
    orc_bloom_contains_policy(words, nblocks, 8, 8, keys, kb, n, seed, out, 1);
}

void orc_bloom_contains_parallel(const uint32_t* words, uint64_t nblocks, const void* keys, uint32_t kb, uint64_t n,
                                 uint64_t seed, uint8_t* out, int threads)
{
    orc_bloom_contains_policy(words, nblocks, 8, 8, keys, kb, n, seed, out, threads);
}

/* ------------------------------------------------------------------------ */
/* HyperLogLog                                                               */
/* ------------------------------------------------------------------------ */

/* HyperLogLogRef::Add (hyperloglog_ref.h:30-47): xxh64 seed 0; index = top p
 * bits; rank = clz(tail) + 1 with a sentinel bit capping it at 65 - p. */
static inline void hll_one(uint8_t* reg, uint32_t p, const uint8_t* key, uint32_t kb)
{
    uint64_t h = orc_xxh64(key, kb, 0);
    uint32_t idx = (uint32_t)(h >> (64 - p));
    uint64_t tail = (h << p) | (1ull << (p - 1));
    uint8_t rank = (uint8_t)(__builtin_clzll(tail) + 1);
    if (reg[idx] < rank) reg[idx] = rank;
}

void orc_hll_add(uint8_t* reg, uint32_t p, const void* keys, uint32_t kb, uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i) hll_one(reg, p, (const uint8_t*)keys + i * kb, kb);
}

/* Per-thread private sketches then a bytewise max -- the same combination rule
 * as the reference's private-sketch Add path (hyperloglog/kernels.h:324-396). */
void orc_hll_add_parallel(uint8_t* reg, uint32_t p, const void* keys, uint32_t kb, uint64_t n, int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
    {
        uint8_t* priv = (uint8_t*)calloc((size_t)1 << p, 1);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i) hll_one(priv, p, (const uint8_t*)keys + (uint64_t)i * kb, kb);
#pragma omp critical
        for (size_t r = 0; r < ((size_t)1 << p); ++r)
            if (reg[r] < priv[r]) reg[r] = priv[r];
        free(priv);
    }
#else
    orc_hll_add(reg, p, keys, kb, n);
#endif
    (void)threads;
}

/* Merge = bytewise max (hyperloglog/kernels.h:55-73). */
void orc_hll_merge(uint8_t* dst, const uint8_t* src, uint32_t p)
{
    for (size_t r = 0; r < ((size_t)1 << p); ++r)
        if (dst[r] < src[r]) dst[r] = src[r];
}

/* HistogramKernel (hyperloglog/kernels.h:74-99): 65 rank bins. */
void orc_hll_histogram(const uint8_t* reg, uint32_t p, uint32_t hist[65])
{
    memset(hist, 0, 65 * sizeof(uint32_t));
    for (size_t r = 0; r < ((size_t)1 << p); ++r) hist[reg[r] < 65 ? reg[r] : 64]++;
}

/* HyperLogLog::Estimate (hyperloglog.inl:327-345) and Finalizer
 * (detail/hyperloglog/finalizer.h:46-151): z = sum hist[r] 2^-r in rank
 * order, then HLL++ (linear counting, threshold, 6-nearest bias interpolation). */
uint64_t orc_hll_finalize(uint32_t p, const uint32_t hist[65], const double* raw, const double* bias, int np,
                          double threshold)
{
    double z = 0.0;
    for (int r = 0; r < 65; ++r) z += ldexp((double)hist[r], -r);
    int v = (int)hist[0];
    int m = 1 << p;
    if (z == 0.0) return UINT64_MAX;
    double alpha;
    switch (m) {
        case 16: alpha = 0.673; break;
        case 32: alpha = 0.697; break;
        case 64: alpha = 0.709; break;
        default: alpha = 0.7213 / (1.0 + 1.079 / m);
    }
    double e = alpha * m * m / z;
    int bias_needed = 0;
    if (v > 0) {
        double h = m * log((double)m / v);
        if (e <= 2.5 * m) return (uint64_t)round(h);
        if (p < 19) {
            if (h <= threshold) e = h;
            else bias_needed = 1;
        }
    } else if (p < 19) {
        bias_needed = 1;
    }
    if (bias_needed && e < 5.0 * m) {
        /* interpolation anchor: binary search, insertion point when absent */
        int left = 0, right = np - 1, anchor = -1, hit = 0;
        while (left <= right) {
            int mid = left + (right - left) / 2;
            if (raw[mid] < e) left = mid + 1;
            else if (raw[mid] > e) right = mid - 1;
            else { anchor = mid; hit = 1; break; }
        }
        if (!hit) anchor = left;
        const int k = 6;
        int low = anchor - k + 1;
        if (low > np - k) low = np - k;
        if (low < 0) low = 0;
        int high = low + k < np ? low + k : np;
        while (high < np && (e - raw[high]) * (e - raw[high]) < (e - raw[low]) * (e - raw[low])) {
            ++low;
            ++high;
        }
        double sum = 0.0;
        for (int i = low; i < high; ++i) sum += bias[i];
        e = e - sum / (high - low);
    }
    if (e >= 18446744073709551615.0) return UINT64_MAX;
    return (uint64_t)round(e);
}
