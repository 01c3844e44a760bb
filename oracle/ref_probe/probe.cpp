// Exposes the reference's own host-compilable math (hash functors, probing
// iterator, capacity rule, Bloom policy, HLL++ finalizer) through a C ABI so
// tests/golden/make_golden.py can record their outputs as fixtures.  Compiled
// from the reference's headers in place by oracle/ref_probe/Makefile; nothing
// of the reference is copied into this repository.
#include <cstdint>
#include <cstring>
#include <stdexcept>

#include "hash_functions.h"
#include "probing_scheme.h"
#include "extent.h"
#include "bloom_filter_policy.h"
#include "detail/hyperloglog/finalizer.h"
#include "roaring_bitmap_ref.h"
#include "utility/equal_wrapper.h"
#include "utility/math_utils.h"

namespace {
template <int B>
struct St { static constexpr int32_t bucketSize = B; };

template <int B>
static uint64_t cap_dh(uint64_t req)
{
    using P = aclco::DoubleHashing<aclco::xxhash_32<uint32_t>>;
    return aclco::MakeValidExtent<P, St<B>>(aclco::Extent<std::size_t>{req});
}
template <int B>
static uint64_t cap_lp(uint64_t req)
{
    using P = aclco::LinearProbing<aclco::xxhash_32<uint32_t>>;
    return aclco::MakeValidExtent<P, St<B>>(aclco::Extent<std::size_t>{req});
}
// First `count` probe indices of a key under the reference's iterator.
template <typename Key, int B>
static void walk(int dh, int hash, Key key, uint32_t cap, uint32_t count, uint32_t* out)
{
    auto run = [&](auto scheme) {
        auto it = scheme.template MakeIterator<B>(key, cap);
        for (uint32_t i = 0; i < count; ++i) { out[i] = *it; ++it; }
    };
    if (hash == 0) {
        if (dh) run(aclco::DoubleHashing<aclco::xxhash_32<Key>>{}); else run(aclco::LinearProbing<aclco::xxhash_32<Key>>{});
    } else if (hash == 1) {
        if (dh) run(aclco::DoubleHashing<aclco::murmurhash3_32<Key>>{}); else run(aclco::LinearProbing<aclco::murmurhash3_32<Key>>{});
    } else if (hash == 2) {
        if constexpr (sizeof(Key) == 2) {
            // the Fmix hashes static_assert 4- or 8-byte keys (utils.h:42-66): no walk
        } else if constexpr (sizeof(Key) == 4) {
            if (dh) run(aclco::DoubleHashing<aclco::murmurhash3_fmix32<Key>>{}); else run(aclco::LinearProbing<aclco::murmurhash3_fmix32<Key>>{});
        } else {
            if (dh) run(aclco::DoubleHashing<aclco::murmurhash3_fmix64<Key>>{}); else run(aclco::LinearProbing<aclco::murmurhash3_fmix64<Key>>{});
        }
    } else {
        if (dh) run(aclco::DoubleHashing<aclco::xxhash_64<Key>>{}); else run(aclco::LinearProbing<aclco::xxhash_64<Key>>{});
    }
}
// The reference's key comparison for floating-point keys, on bit patterns:
// EqualWrapper<T, EqualTo<T>> (utility/equal_wrapper.h) returns 1 for EQUAL
// from EqualTo and, from IsSentinelValue, whether the value is the sentinel.
template <typename T, typename Bits>
static int eq_of(Bits a, Bits b, int sentinel)
{
    T x, y;
    std::memcpy(&x, &a, sizeof(T));
    std::memcpy(&y, &b, sizeof(T));
    aclco::EqualWrapper<T, aclco::EqualTo<T>> w{aclco::EqualTo<T>{}};
    if (sentinel) return w.IsSentinelValue(x, y) ? 1 : 0;
    return w.EqualTo(x, y) == aclco::EqualResult::EQUAL ? 1 : 0;
}
}  // namespace

extern "C" {
uint32_t ref_xxh32_u32(uint32_t k, uint32_t seed) { return aclco::xxhash_32<uint32_t>{seed}(k); }
uint32_t ref_xxh32_u64(uint64_t k, uint32_t seed) { return aclco::xxhash_32<uint64_t>{seed}(k); }
uint64_t ref_xxh64_u32(uint32_t k, uint64_t seed) { return aclco::xxhash_64<uint32_t>{seed}(k); }
uint64_t ref_xxh64_u64(uint64_t k, uint64_t seed) { return aclco::xxhash_64<uint64_t>{seed}(k); }
uint64_t ref_xxh64_i64(int64_t k, uint64_t seed) { return aclco::xxhash_64<int64_t>{seed}(k); }
uint64_t ref_xxh64_f32(float k, uint64_t seed) { return aclco::xxhash_64<float>{seed}(k); }
uint32_t ref_murmur3_u32(uint32_t k, uint32_t seed) { return aclco::murmurhash3_32<uint32_t>{seed}(k); }
uint32_t ref_murmur3_u64(uint64_t k, uint32_t seed) { return aclco::murmurhash3_32<uint64_t>{seed}(k); }
uint32_t ref_fmix32(uint32_t k, uint32_t seed) { return aclco::murmurhash3_fmix32<uint32_t>{seed}(k); }
uint32_t ref_xxh32_u16(uint16_t k, uint32_t seed) { return aclco::xxhash_32<uint16_t>{seed}(k); }
uint32_t ref_murmur3_u16(uint16_t k, uint32_t seed) { return aclco::murmurhash3_32<uint16_t>{seed}(k); }
uint64_t ref_xxh64_u16(uint16_t k, uint64_t seed) { return aclco::xxhash_64<uint16_t>{seed}(k); }

int ref_equal_f16(uint16_t a, uint16_t b, int sentinel) { return eq_of<_Float16>(a, b, sentinel); }
int ref_equal_f32(uint32_t a, uint32_t b, int sentinel) { return eq_of<float>(a, b, sentinel); }
int ref_equal_f64(uint64_t a, uint64_t b, int sentinel) { return eq_of<double>(a, b, sentinel); }
uint64_t ref_fmix64(uint64_t k, uint64_t seed) { return aclco::murmurhash3_fmix64<uint64_t>{seed}(k); }

uint64_t ref_prime_count() { return aclco::primes.size(); }
int64_t ref_prime_at(uint64_t i) { return aclco::primes[i]; }

// Returns 0 when the reference throws.
uint64_t ref_valid_capacity(uint64_t req, int b, int dh)
{
    try {
        switch (b) {
            case 1: return dh ? cap_dh<1>(req) : cap_lp<1>(req);
            case 2: return dh ? cap_dh<2>(req) : cap_lp<2>(req);
            case 4: return dh ? cap_dh<4>(req) : cap_lp<4>(req);
            case 5: return dh ? cap_dh<5>(req) : cap_lp<5>(req);
            case 8: return dh ? cap_dh<8>(req) : cap_lp<8>(req);
        }
    } catch (std::exception const&) {
    }
    return 0;
}

void ref_probe_walk(int key_bytes, int b, int dh, int hash, uint64_t key, uint32_t cap, uint32_t count, uint32_t* out)
{
    if (key_bytes == 2) {
        uint16_t k = static_cast<uint16_t>(key);
        switch (b) {
            case 1: walk<uint16_t, 1>(dh, hash, k, cap, count, out); break;
            case 5: walk<uint16_t, 5>(dh, hash, k, cap, count, out); break;
            case 8: walk<uint16_t, 8>(dh, hash, k, cap, count, out); break;
        }
    } else if (key_bytes == 4) {
        uint32_t k = static_cast<uint32_t>(key);
        switch (b) {
            case 1: walk<uint32_t, 1>(dh, hash, k, cap, count, out); break;
            case 5: walk<uint32_t, 5>(dh, hash, k, cap, count, out); break;
            case 8: walk<uint32_t, 8>(dh, hash, k, cap, count, out); break;
        }
    } else {
        switch (b) {
            case 1: walk<uint64_t, 1>(dh, hash, key, cap, count, out); break;
            case 5: walk<uint64_t, 5>(dh, hash, key, cap, count, out); break;
            case 8: walk<uint64_t, 8>(dh, hash, key, cap, count, out); break;
        }
    }
}

// Default Bloom policy: block index and the 8 word patterns of one key.
void ref_bloom_locate(int key_bytes, uint64_t key, uint64_t num_blocks, uint64_t seed, uint32_t* block,
                      uint32_t* patterns)
{
    auto go = [&](auto k) {
        using K = decltype(k);
        aclco::BloomFilterPolicy<K> pol{aclco::xxhash_64<K>{seed}};
        uint64_t h = pol.HashKey(k);
        *block = pol.BlockIndex(static_cast<uint32_t>(h >> 32), num_blocks);
        for (uint32_t w = 0; w < 8; ++w) patterns[w] = pol.WordPatternForLane(w, static_cast<uint32_t>(h));
    };
    if (key_bytes == 4) go(static_cast<uint32_t>(key)); else go(key);
}

}  // extern "C"

namespace {
template <uint32_t W, uint32_t P>
int locate_policy(int key_bytes, uint64_t key, uint64_t num_blocks, uint64_t seed, uint32_t* block,
                  uint32_t* patterns)
{
    auto go = [&](auto k) {
        using K = decltype(k);
        aclco::BloomFilterPolicy<K, aclco::xxhash_64<K>, uint32_t, W, P> pol{aclco::xxhash_64<K>{seed}};
        uint64_t h = pol.HashKey(k);
        *block = pol.BlockIndex(static_cast<uint32_t>(h >> 32), num_blocks);
        for (uint32_t w = 0; w < W; ++w) patterns[w] = pol.WordPatternForLane(w, static_cast<uint32_t>(h));
    };
    if (key_bytes == 4) go(static_cast<uint32_t>(key)); else go(key);
    return 0;
}
}  // namespace

extern "C" {

// Any of the policies the fixtures cover: block index and the W word patterns of one key.
int ref_bloom_locate_policy(int key_bytes, uint64_t key, uint64_t num_blocks, uint64_t seed, uint32_t words_per_block,
                            uint32_t pattern_bits, uint32_t* block, uint32_t* patterns)
{
#define B2CO_POLICY(W, P) \
    if (words_per_block == W && pattern_bits == P) return locate_policy<W, P>(key_bytes, key, num_blocks, seed, block, patterns);
    B2CO_POLICY(1, 1)
    B2CO_POLICY(1, 32)
    B2CO_POLICY(2, 2)
    B2CO_POLICY(2, 64)
    B2CO_POLICY(4, 4)
    B2CO_POLICY(4, 16)
    B2CO_POLICY(8, 8)
    B2CO_POLICY(8, 16)
    B2CO_POLICY(8, 64)
    B2CO_POLICY(16, 16)
    B2CO_POLICY(16, 48)
    B2CO_POLICY(32, 32)
    B2CO_POLICY(32, 64)
#undef B2CO_POLICY
    return -1;
}

// Roaring portable format: the reference's host parser (bounded by `bytes`),
// then its membership query compiled for the host.  Returns 0, or 1 when the
// parser rejects the input (the reference's std::invalid_argument).
int ref_roaring(int key64, uint8_t const* data, uint64_t bytes, uint64_t const* keys, uint64_t n, uint8_t* out,
                uint64_t* num_keys, uint64_t* size_bytes)
{
    try {
        if (key64) {
            auto parsed = aclco::detail::ParseRoaringBitmap<uint64_t>(data, bytes);
            aclco::RoaringBitmapRef<uint64_t> ref(data, &parsed.metadata, parsed.buckets.data(),
                                                  parsed.metadata.numKeys, parsed.metadata.sizeBytes);
            for (uint64_t i = 0; i < n; ++i) out[i] = ref.Contains(keys[i]);
            *num_keys = parsed.metadata.numKeys;
            *size_bytes = parsed.metadata.sizeBytes;
        } else {
            auto parsed = aclco::detail::ParseRoaringBitmap<uint32_t>(data, bytes);
            aclco::RoaringBitmapRef<uint32_t> ref(data, &parsed.metadata, parsed.metadata.numKeys,
                                                  parsed.metadata.sizeBytes);
            for (uint64_t i = 0; i < n; ++i) out[i] = ref.Contains(static_cast<uint32_t>(keys[i]));
            *num_keys = parsed.metadata.numKeys;
            *size_bytes = parsed.metadata.sizeBytes;
        }
    } catch (std::invalid_argument const&) {
        return 1;
    }
    return 0;
}

uint64_t ref_hll_finalize(int precision, double z, int v)
{
    return aclco::detail::hyperloglog::Finalizer(precision)(z, v);
}
// The finalizer's interpolation data (raw estimates, biases, threshold).
int ref_hll_points(int p) { return static_cast<int>(aclco::detail::hyperloglog::raw_estimate_data_size(p)); }
double ref_hll_raw(int p, int i) { return aclco::detail::hyperloglog::raw_estimate_data(p)[i]; }
double ref_hll_bias(int p, int i) { return aclco::detail::hyperloglog::bias_data(p)[i]; }
double ref_hll_threshold(int p) { return aclco::detail::hyperloglog::threshold(p); }
}
