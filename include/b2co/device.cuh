// device.cuh -- the hashing, probing and slot primitives of the b2co tables,
// usable from device code a caller compiles with nvcc (ForEach callbacks in
// for_each.cuh) and shared with the library's own kernels.
//
// Semantics follow the reference (ops-collections) exactly; each piece cites
// the reference file it restates.  Everything here is __host__ __device__ so
// the same code is unit-tested on the CPU.
#pragma once

#include <cstddef>
#include <cstdint>
#include <type_traits>

#include <cuda_runtime.h>

#include "../b2co.h"

#define B2CO_HD __host__ __device__ __forceinline__

namespace b2co {

// ---------------------------------------------------------------------------
// hashes over a key's object representation (little-endian, 2, 4 or 8 bytes)
// ---------------------------------------------------------------------------

B2CO_HD uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
B2CO_HD uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

// XXH32 for 2-, 4- and 8-byte inputs (include/detail/hash_functions/xxhash.h:52-175:
// inputs shorter than 16 bytes take the seed+prime5 start, then 4-byte lanes,
// then single bytes).
template <int KB>
B2CO_HD uint32_t xxh32(uint64_t key, uint32_t seed)
{
    constexpr uint32_t P1 = 0x9e3779b1u, P2 = 0x85ebca77u, P3 = 0xc2b2ae3du, P4 = 0x27d4eb2fu, P5 = 0x165667b1u;
    uint32_t h = seed + P5 + uint32_t(KB);
    if constexpr (KB == 2) {
        h = rotl32(h + uint32_t(key & 0xffu) * P5, 11) * P1;
        h = rotl32(h + uint32_t((key >> 8) & 0xffu) * P5, 11) * P1;
    } else {
        h = rotl32(h + uint32_t(key) * P3, 17) * P4;
        if constexpr (KB == 8) h = rotl32(h + uint32_t(key >> 32) * P3, 17) * P4;
    }
    h ^= h >> 15;
    h *= P2;
    h ^= h >> 13;
    h *= P3;
    h ^= h >> 16;
    return h;
}

// XXH64 for 2-, 4- and 8-byte inputs (xxhash.h:184-326, fast paths :199-218,
// single trailing bytes after them).
template <int KB>
B2CO_HD uint64_t xxh64(uint64_t key, uint64_t seed)
{
    constexpr uint64_t P1 = 11400714785074694791ull, P2 = 14029467366897019727ull, P3 = 1609587929392839161ull,
                       P4 = 9650029242287828579ull, P5 = 2870177450012600261ull;
    uint64_t h = seed + P5 + uint64_t(KB);
    if constexpr (KB == 8) {
        h ^= rotl64(key * P2, 31) * P1;
        h = rotl64(h, 27) * P1 + P4;
    } else if constexpr (KB == 2) {
        h ^= uint64_t(key & 0xffu) * P5;
        h = rotl64(h, 11) * P1;
        h ^= uint64_t((key >> 8) & 0xffu) * P5;
        h = rotl64(h, 11) * P1;
    } else {
        h ^= uint64_t(uint32_t(key)) * P1;
        h = rotl64(h, 23) * P2 + P3;
    }
    h ^= h >> 33;
    h *= P2;
    h ^= h >> 29;
    h *= P3;
    h ^= h >> 32;
    return h;
}

// MurmurHash3 finalizers with the seed xor-ed in first (hash_functions/utils.h:42-66).
B2CO_HD uint32_t fmix32(uint32_t k, uint32_t seed)
{
    uint32_t h = k ^ seed;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
B2CO_HD uint64_t fmix64(uint64_t k, uint64_t seed)
{
    uint64_t h = k ^ seed;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return h;
}

// MurmurHash3_x86_32 for 2-, 4- and 8-byte inputs (hash_functions/murmurhash3.h:57-106).
template <int KB>
B2CO_HD uint32_t murmur3_32(uint64_t key, uint32_t seed)
{
    constexpr uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    uint32_t h = seed;
#pragma unroll
    for (int i = 0; i < KB / 4; ++i) {
        uint32_t k = uint32_t(key >> (32 * i));
        k *= c1;
        k = rotl32(k, 15);
        k *= c2;
        h ^= k;
        h = rotl32(h, 13);
        h = h * 5 + 0xe6546b64u;
    }
    if constexpr (KB == 2) {  // the two tail bytes
        uint32_t k = uint32_t(key & 0xffffu);
        k *= c1;
        k = rotl32(k, 15);
        k *= c2;
        h ^= k;
    }
    h ^= uint32_t(KB);
    return fmix32(h, 0);
}

// The probing schemes cast the hash to the kernels' uint32 size type
// (utility/math_utils.h:14-24 SanitizeHash).  The Fmix family takes 4- and
// 8-byte keys only (utils.h:42-66 static_asserts the size); tables refuse it
// for other widths.
template <int KB>
B2CO_HD uint32_t probe_hash(uint32_t kind, uint64_t key, uint32_t seed)
{
    switch (kind) {
        case B2CO_HASH_MURMUR3_32: return murmur3_32<KB>(key, seed);
        case B2CO_HASH_FMIX:
            if constexpr (KB == 4) return fmix32(uint32_t(key), seed);
            else if constexpr (KB == 8) return uint32_t(fmix64(key, seed));
            else return 0;
        case B2CO_HASH_XXH64: return uint32_t(xxh64<KB>(key, seed));
        default: return xxh32<KB>(key, seed);
    }
}

// ---------------------------------------------------------------------------
// exact 32-bit remainder by a runtime divisor (Lemire, Kaser, Kurz, "Faster
// remainder by direct computation", 2019): M = floor((2^64-1)/d) + 1 and
// a mod d = mulhi64(M * a, d) for every 32-bit a and d >= 1.
// ---------------------------------------------------------------------------

struct FastMod {
    uint64_t m;
    uint32_t d;
};
inline FastMod make_fastmod(uint32_t d) { return FastMod{~0ull / d + 1ull, d}; }

B2CO_HD uint64_t mulhi64(uint64_t a, uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return uint64_t((unsigned __int128)a * b >> 64);
#endif
}
B2CO_HD uint32_t fastmod(uint32_t a, FastMod f) { return uint32_t(mulhi64(f.m * uint64_t(a), f.d)); }

// ---------------------------------------------------------------------------
// probing: LinearProbing / DoubleHashing iterators
// (detail/probing_scheme/probing_scheme_impl.inl:24-91, 116-128, 175-189)
// ---------------------------------------------------------------------------

struct ProbeParams {
    uint32_t capacity;   // slots (a multiple of the bucket size)
    uint32_t nbuckets;   // capacity / bucket size
    FastMod mod_nb;      // % nbuckets
    FastMod mod_nbm1;    // % (nbuckets - 1), double hashing only
    uint32_t probing;    // B2CO_PROBE_*
    uint32_t hash;       // B2CO_HASH_*
};

// Probe parameters of a table of `capacity` slots in buckets of `bucket_size`.
inline ProbeParams make_probe_params(uint64_t capacity, uint32_t bucket_size, uint32_t probing, uint32_t hash)
{
    ProbeParams p{};
    p.capacity = uint32_t(capacity);
    p.nbuckets = uint32_t(capacity / bucket_size);
    p.mod_nb = make_fastmod(p.nbuckets);
    p.mod_nbm1 = make_fastmod(p.nbuckets > 1 ? p.nbuckets - 1 : 1);
    p.probing = probing;
    p.hash = hash;
    return p;
}

template <int KB, int B>
B2CO_HD uint32_t probe_init(ProbeParams const& p, uint64_t key)
{
    return fastmod(probe_hash<KB>(p.hash, key, 0), p.mod_nb) * uint32_t(B);
}

// DoubleHashing's second hash is the same family seeded with 1 (probing_scheme.h:99).
template <int KB, int B>
B2CO_HD uint32_t probe_step(ProbeParams const& p, uint64_t key)
{
    if (p.probing == B2CO_PROBE_LINEAR) return uint32_t(B);
    return (fastmod(probe_hash<KB>(p.hash, key, 1), p.mod_nbm1) + 1u) * uint32_t(B);
}

// Subtract before adding so the wrap never overflows (probing_scheme_impl.inl:76-84).
B2CO_HD uint32_t probe_next(uint32_t idx, uint32_t step, uint32_t capacity)
{
    uint32_t rem = capacity - step;
    return idx >= rem ? idx - rem : idx + step;
}

// ---------------------------------------------------------------------------
// slot layouts: Pair<K,V> aligned to min(16, bitceil(sizeof K + sizeof V))
// (pair.h:41, pair.inl:19-24), or a bare key for sets
// ---------------------------------------------------------------------------

struct alignas(16) U128 {
    uint64_t lo, hi;
};

// Key equality (KeyEqual = EqualTo, utility/math_utils.h:66-70, applied by
// equal_wrapper.h:30-33).  Integer keys compare their bits.  Floating-point
// keys (fp16, fp32, fp64 by width) compare as IEEE values: -0 equals +0 and a
// NaN equals nothing, itself included.  Sentinel tests stay bitwise
// (equal_wrapper.h:35-42 with traits.h:27-28), so they never call this.
template <int KB, bool FLOAT_KEY>
B2CO_HD bool key_equal(uint64_t a, uint64_t b)
{
    if constexpr (!FLOAT_KEY) {
        return a == b;
    } else {
        constexpr uint64_t sign = 1ull << (8 * KB - 1);
        constexpr uint64_t inf = KB == 2 ? 0x7c00ull : (KB == 4 ? 0x7f800000ull : 0x7ff0000000000000ull);
        uint64_t const ma = a & ~sign, mb = b & ~sign;  // magnitudes (keys arrive masked to KB bytes)
        if (ma > inf || mb > inf) return false;         // a NaN on either side
        return a == b || (ma | mb) == 0;                 // same value, or +0 against -0
    }
}

// A slot: Pair<K,V> aligned to min(16, bitceil(sizeof K + sizeof V)) with the
// payload at the next offset aligned to its own size, or a bare key for sets.
// FLOAT_KEY selects IEEE key equality (fp16/fp32/fp64 keys by width).
template <int KB, int VB, bool FLOAT_KEY = false>
struct SlotT {
    static constexpr int key_bytes = KB;
    static constexpr int value_bytes = VB;
    static constexpr bool is_set = VB == 0;
    static constexpr bool float_key = FLOAT_KEY;
    static constexpr int value_offset = VB == 0 ? 0 : ((KB + VB - 1) / VB) * VB;
    static constexpr int pair_align = (KB + VB) <= 4 ? 4 : ((KB + VB) <= 8 ? 8 : 16);
    static constexpr int bytes = VB == 0 ? KB : ((value_offset + VB + pair_align - 1) / pair_align) * pair_align;
    // raw storage word of one slot
    using Raw = typename std::conditional<bytes == 2, unsigned short,
                typename std::conditional<bytes == 4, uint32_t,
                typename std::conditional<bytes == 8, unsigned long long, U128>::type>::type>::type;
    static constexpr uint64_t kmask = KB == 8 ? ~0ull : ((1ull << (8 * KB)) - 1ull);
    static constexpr uint64_t vmask = VB == 8 ? ~0ull : (VB == 0 ? 0ull : ((1ull << (8 * VB)) - 1ull));

    B2CO_HD static bool key_eq(uint64_t a, uint64_t b) { return key_equal<KB, FLOAT_KEY>(a, b); }

    B2CO_HD static uint64_t key(Raw r)
    {
        if constexpr (bytes == 16) return r.lo & kmask;
        else return uint64_t(r) & kmask;
    }
    // Payload; a set's payload is the stored key (open_addressing_ref_impl.h:71-79).
    B2CO_HD static uint64_t value(Raw r)
    {
        if constexpr (is_set) return key(r);
        else if constexpr (bytes == 16) return r.hi & vmask;  // 16-byte pairs keep the payload at offset 8
        else return (uint64_t(r) >> (8 * value_offset)) & vmask;
    }
    B2CO_HD static Raw make(uint64_t k, uint64_t v)
    {
        if constexpr (bytes == 16) {
            U128 r;
            r.lo = k & kmask;
            r.hi = v & vmask;
            return r;
        } else if constexpr (is_set) {
            return Raw(k & kmask);
        } else {
            return Raw((k & kmask) | ((v & vmask) << (8 * value_offset)));
        }
    }
    // Same slot with the key replaced, every other byte kept.
    B2CO_HD static Raw with_key(Raw r, uint64_t k)
    {
        if constexpr (bytes == 16) {
            r.lo = (r.lo & ~kmask) | (k & kmask);
            return r;
        } else if constexpr (!is_set) {
            return Raw((uint64_t(r) & ~kmask) | (k & kmask));
        } else {
            return Raw(k & kmask);
        }
    }
};

B2CO_HD bool raw_eq(unsigned short a, unsigned short b) { return a == b; }
B2CO_HD bool raw_eq(uint32_t a, uint32_t b) { return a == b; }
B2CO_HD bool raw_eq(unsigned long long a, unsigned long long b) { return a == b; }
B2CO_HD bool raw_eq(U128 a, U128 b) { return a.lo == b.lo && a.hi == b.hi; }

}  // namespace b2co
