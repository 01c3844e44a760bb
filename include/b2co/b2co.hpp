// b2co.hpp -- C++ mirror of the ops-collections container API over libb2co.so.
//
// A C++ caller of the reference switches by replacing `aclco::` with `b2co::`,
// `aclrtStream` with `cudaStream_t` and the reference headers with this one:
// class templates, method names, argument order and meaning, return values
// and exception types follow the reference headers (include/static_map.h,
// static_set.h, dynamic_map.h, bloom_filter.h, hyperloglog.h, hash_functions.h,
// probing_scheme.h, storage.h, extent.h, pair.h).  The work itself runs in the
// library's sm_100a kernels behind the C ABI (include/b2co.h).
//
// Compile-time policy types select run-time descriptor fields.  Predicates
// cannot cross a C ABI: they are limited to AlwaysTrue and the `uint8_t != 0`
// stencil.  ForEach callbacks run in a kernel template compiled by the
// caller's nvcc (b2co/for_each.cuh, pulled in when this header is compiled as
// CUDA): StaticMap / StaticSet have ForEach / ForEachAsync only there.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include <cuda_fp16.h>
#include <cuda_runtime_api.h>

#include "../b2co.h"

namespace b2co {

// ---- errors: status codes back to the reference's exception types ----------
inline void throw_on(int status)
{
    if (status == B2CO_OK) return;
    std::string msg = b2co_last_error();
    switch (status) {
        case B2CO_EINVAL: throw std::invalid_argument(msg);
        case B2CO_ERANGE: throw std::length_error(msg);
        case B2CO_ENOMEM: throw std::bad_alloc();
        case B2CO_ELOGIC: throw std::logic_error(msg);
        case B2CO_EOVERFLOW: throw std::overflow_error(msg);
        default: throw std::runtime_error(msg);
    }
}

inline b2co_stream to_stream(cudaStream_t s) { return reinterpret_cast<b2co_stream>(s); }

// ---- hash_functions.h ------------------------------------------------------
namespace detail {
template <int Kind, typename Key>
struct HashTag {
    static constexpr int kind = Kind;
    using ArgumentType = Key;
    constexpr HashTag(uint32_t seed = 0) : seed_{seed} {}
    constexpr bool operator==(HashTag const& o) const { return seed_ == o.seed_; }
    uint32_t seed_;
};
}  // namespace detail
template <typename Key> using xxhash_32 = detail::HashTag<B2CO_HASH_XXH32, Key>;
template <typename Key> using murmurhash3_32 = detail::HashTag<B2CO_HASH_MURMUR3_32, Key>;
template <typename Key> using murmurhash3_fmix32 = detail::HashTag<B2CO_HASH_FMIX, Key>;
template <typename Key> using murmurhash3_fmix64 = detail::HashTag<B2CO_HASH_FMIX, Key>;
template <typename Key> using xxhash_64 = detail::HashTag<B2CO_HASH_XXH64, Key>;

// ---- probing_scheme.h / storage.h / extent.h / pair.h ------------------------
template <class Hash>
struct LinearProbing {
    static constexpr uint32_t probing = B2CO_PROBE_LINEAR;
    static constexpr uint32_t hash = Hash::kind;
    constexpr LinearProbing(Hash const& h = {}) : hash_{h} {}
    constexpr bool operator==(LinearProbing const& o) const { return hash_ == o.hash_; }
    Hash hash_;
};
// The second hash defaults to the first family seeded with 1 (probing_scheme.h:99).
template <class Hash1, class Hash2 = Hash1>
struct DoubleHashing {
    static_assert(Hash1::kind == Hash2::kind, "both hashes of DoubleHashing must be the same family");
    static constexpr uint32_t probing = B2CO_PROBE_DOUBLE;
    static constexpr uint32_t hash = Hash1::kind;
    constexpr DoubleHashing(Hash1 const& h1 = {}, Hash2 const& h2 = {1}) : h1_{h1}, h2_{h2} {}
    constexpr bool operator==(DoubleHashing const& o) const { return h1_ == o.h1_ && h2_ == o.h2_; }
    Hash1 h1_;
    Hash2 h2_;
};

template <int32_t BucketSize>
struct Storage {
    static constexpr int32_t bucketSize = BucketSize;
};

template <typename SizeType = std::size_t>
struct Extent {
    using ValueType = SizeType;
    constexpr Extent(SizeType s) : size_{s} {}
    constexpr operator SizeType() const { return size_; }
    SizeType size_;
};

template <typename T>
struct EqualTo {
    constexpr bool operator==(EqualTo const&) const { return true; }
};

struct AlwaysTrue {};

constexpr std::size_t pair_alignment(std::size_t bytes)
{
    std::size_t a = 1;
    while (a < bytes) a <<= 1;
    return a < 16 ? a : 16;
}
template <typename First, typename Second>
struct alignas(pair_alignment(sizeof(First) + sizeof(Second))) Pair {
    First first;
    Second second;
};

// The reference's fp16_t key / payload type (2 bytes, IEEE binary16).
using fp16_t = __half;

namespace detail {

// Floating-point keys (float, double, fp16_t) match with == in the reference
// (EqualTo); the table is created with that key kind.
template <typename T>
constexpr bool is_float_key = std::is_floating_point<T>::value || std::is_same<T, __half>::value;

template <typename T>
uint64_t bits_of(T v)
{
    uint64_t b = 0;
    std::memcpy(&b, &v, sizeof(T));
    return b;
}

#if defined(__CUDACC__)
// Defined in b2co/for_each.cuh (T = void for a set).
template <class CallbackOp, class Key, class T>
void for_each_async(b2co_oa_table* t, void* keys, uint64_t n, void* args, cudaStream_t stream);
#endif

// Instance state of probing schemes / KeyEqual cannot reach the device
// (open_addressing_impl.h:40-49 rejects non-default instances).
template <typename T>
void validate_default(T const& v, char const* name)
{
    if (!(v == T{})) throw std::invalid_argument(std::string(name) + " carries instance state that cannot take effect on device");
}

template <class Key, class T, class ExtentT, class KeyEqual, class ProbingScheme, class StorageT>
class OpenAddressing {
   public:
    using SizeType = typename ExtentT::ValueType;
    static constexpr int32_t bucketSize = StorageT::bucketSize;

    OpenAddressing(ExtentT capacity, Key emptyKey, T emptyValue, Key erasedKey, std::size_t valueBytes,
                   KeyEqual const& pred, ProbingScheme const& probing, cudaStream_t stream)
    {
        validate_default(probing, "ProbingScheme");
        validate_default(pred, "KeyEqual");
        b2co_oa_desc d{};
        d.key_bytes = sizeof(Key);
        d.value_bytes = uint32_t(valueBytes);
        d.bucket_size = bucketSize;
        d.probing = ProbingScheme::probing;
        d.hash = ProbingScheme::hash;
        d.key_kind = is_float_key<Key> ? B2CO_KEY_FLOAT : B2CO_KEY_INTEGER;
        d.empty_key_bits = bits_of(emptyKey);
        d.empty_value_bits = valueBytes ? bits_of(emptyValue) : 0;
        d.erased_key_bits = bits_of(erasedKey);
        throw_on(b2co_oa_create(&d, static_cast<SizeType>(capacity), to_stream(stream), &t_));
    }
    ~OpenAddressing() { b2co_oa_destroy(t_); }
    OpenAddressing(OpenAddressing const&) = delete;
    OpenAddressing& operator=(OpenAddressing const&) = delete;
    OpenAddressing(OpenAddressing&& o) noexcept : t_{std::exchange(o.t_, nullptr)} {}
    OpenAddressing& operator=(OpenAddressing&& o) noexcept
    {
        if (this != &o) {
            b2co_oa_destroy(t_);
            t_ = std::exchange(o.t_, nullptr);
        }
        return *this;
    }

    SizeType Insert(void* v, ExtentT n, cudaStream_t s)
    {
        uint64_t f = 0;
        throw_on(b2co_oa_insert(t_, v, static_cast<SizeType>(n), to_stream(s), &f));
        return SizeType(f);
    }
    void InsertAsync(void* v, ExtentT n, cudaStream_t s) { throw_on(b2co_oa_insert_async(t_, v, static_cast<SizeType>(n), to_stream(s))); }
    template <typename StencilT = uint8_t, typename Predicate = AlwaysTrue>
    SizeType InsertIf(void* v, StencilT* st, ExtentT n, cudaStream_t s)
    {
        static_assert(sizeof(StencilT) == 1, "the C ABI carries uint8 stencils (nonzero = selected)");
        uint64_t f = 0;
        throw_on(b2co_oa_insert_if(t_, v, reinterpret_cast<uint8_t const*>(st), static_cast<SizeType>(n), to_stream(s), &f));
        return SizeType(f);
    }
    template <typename StencilT = uint8_t, typename Predicate = AlwaysTrue>
    void InsertIfAsync(void* v, StencilT* st, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_insert_if_async(t_, v, reinterpret_cast<uint8_t const*>(st), static_cast<SizeType>(n), to_stream(s)));
    }
    void InsertAndFind(void* v, void* of, void* oi, ExtentT n, cudaStream_t s, int mode = B2CO_IAF_RACE)
    {
        throw_on(b2co_oa_insert_and_find(t_, v, of, static_cast<uint8_t*>(oi), static_cast<SizeType>(n), mode, to_stream(s)));
    }
    void InsertAndFindAsync(void* v, void* of, void* oi, ExtentT n, cudaStream_t s, int mode = B2CO_IAF_RACE)
    {
        throw_on(b2co_oa_insert_and_find_async(t_, v, of, static_cast<uint8_t*>(oi), static_cast<SizeType>(n), mode, to_stream(s)));
    }
    SizeType Erase(void* k, ExtentT n, cudaStream_t s)
    {
        uint64_t f = 0;
        throw_on(b2co_oa_erase(t_, k, static_cast<SizeType>(n), to_stream(s), &f));
        return SizeType(f);
    }
    void EraseAsync(void* k, ExtentT n, cudaStream_t s) { throw_on(b2co_oa_erase_async(t_, k, static_cast<SizeType>(n), to_stream(s))); }
    void Clear(cudaStream_t s) { throw_on(b2co_oa_clear(t_, to_stream(s))); }
    void ClearAsync(cudaStream_t s) noexcept { (void)b2co_oa_clear_async(t_, to_stream(s)); }
    void Find(void* k, void* o, ExtentT n, cudaStream_t s) { throw_on(b2co_oa_find(t_, k, o, static_cast<SizeType>(n), to_stream(s))); }
    void FindAsync(void* k, void* o, ExtentT n, cudaStream_t s) { throw_on(b2co_oa_find_async(t_, k, o, static_cast<SizeType>(n), to_stream(s))); }
    template <typename StencilT = uint8_t, typename Predicate = AlwaysTrue>
    void FindIf(void* k, StencilT* st, void* o, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_find_if(t_, k, reinterpret_cast<uint8_t const*>(st), o, static_cast<SizeType>(n), to_stream(s)));
    }
    template <typename StencilT = uint8_t, typename Predicate = AlwaysTrue>
    void FindIfAsync(void* k, StencilT* st, void* o, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_find_if_async(t_, k, reinterpret_cast<uint8_t const*>(st), o, static_cast<SizeType>(n), to_stream(s)));
    }
    void Contains(void* k, void* o, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_contains(t_, k, static_cast<uint8_t*>(o), static_cast<SizeType>(n), to_stream(s)));
    }
    void ContainsAsync(void* k, void* o, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_contains_async(t_, k, static_cast<uint8_t*>(o), static_cast<SizeType>(n), to_stream(s)));
    }
    template <typename StencilT = uint8_t, typename Predicate = AlwaysTrue>
    void ContainsIf(void* k, StencilT* st, void* o, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_contains_if(t_, k, reinterpret_cast<uint8_t const*>(st), static_cast<uint8_t*>(o), static_cast<SizeType>(n), to_stream(s)));
    }
    template <typename StencilT = uint8_t, typename Predicate = AlwaysTrue>
    void ContainsIfAsync(void* k, StencilT* st, void* o, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_contains_if_async(t_, k, reinterpret_cast<uint8_t const*>(st), static_cast<uint8_t*>(o), static_cast<SizeType>(n), to_stream(s)));
    }
    SizeType Count(void* k, ExtentT n, cudaStream_t s)
    {
        uint64_t c = 0;
        throw_on(b2co_oa_count(t_, k, static_cast<SizeType>(n), to_stream(s), &c));
        return SizeType(c);
    }
    SizeType Capacity() const
    {
        uint64_t c = 0;
        throw_on(b2co_oa_capacity(t_, &c));
        return SizeType(c);
    }
    void* Data() const
    {
        void* p = nullptr;
        throw_on(b2co_oa_data(t_, &p));
        return p;
    }
    void SetErased(uint64_t bits, cudaStream_t s) { throw_on(b2co_oa_set_erased_key(t_, bits, to_stream(s))); }
    b2co_oa_table* handle() const { return t_; }

   private:
    b2co_oa_table* t_ = nullptr;
};

}  // namespace detail

// ---- static_map.h ----------------------------------------------------------
template <class Key, class T, class ExtentT = Extent<std::size_t>, class KeyEqual = EqualTo<Key>,
          class ProbingScheme = LinearProbing<murmurhash3_32<Key>>, class StorageT = Storage<5>>
class StaticMap : public detail::OpenAddressing<Key, T, ExtentT, KeyEqual, ProbingScheme, StorageT> {
    static_assert(sizeof(Key) == 2 || sizeof(Key) == 4 || sizeof(Key) == 8, "keys are 2, 4 or 8 bytes");
    static_assert(sizeof(Key) == 2 ? sizeof(T) == 2 : (sizeof(T) == 4 || sizeof(T) == 8),
                  "2-byte keys take 2-byte payloads; wider keys take 4- or 8-byte payloads");
    using Base = detail::OpenAddressing<Key, T, ExtentT, KeyEqual, ProbingScheme, StorageT>;

   public:
    using SizeType = typename Base::SizeType;
    using KeyType = Key;
    using ValueType = Pair<Key, T>;

    StaticMap(ExtentT capacity, Key emptyKey, T emptyValue, KeyEqual const& pred = {},
              ProbingScheme const& probing = {}, StorageT = {}, cudaStream_t stream = nullptr)
        : Base(capacity, emptyKey, emptyValue, emptyKey, sizeof(T), pred, probing, stream), emptyKey_{emptyKey}
    {}
    void SetErasedKey(Key erasedKey, cudaStream_t s) { this->SetErased(detail::bits_of(erasedKey), s); }
    SizeType InsertOrAssign(void* v, ExtentT n, cudaStream_t s)
    {
        SizeType assigned;
        return InsertOrAssign(v, n, s, assigned);
    }
    SizeType InsertOrAssign(void* v, ExtentT n, cudaStream_t s, SizeType& assignedNum)
    {
        uint64_t f = 0, a = 0;
        throw_on(b2co_oa_insert_or_assign(this->handle(), v, static_cast<SizeType>(n), to_stream(s), &f, &a));
        assignedNum = SizeType(a);
        return SizeType(f);
    }
    void InsertOrAssignAsync(void* v, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_insert_or_assign_async(this->handle(), v, static_cast<SizeType>(n), to_stream(s)));
    }
    template <typename StencilT = uint8_t, typename Predicate = AlwaysTrue>
    void AssignIfAsync(void* v, StencilT* st, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_oa_assign_if_async(this->handle(), v, reinterpret_cast<uint8_t const*>(st), static_cast<SizeType>(n), to_stream(s)));
    }
    ValueType* Data() const { return static_cast<ValueType*>(Base::Data()); }
#if defined(__CUDACC__)
    // reference: static_map.h:533-558 ForEach / ForEachAsync (static_map.inl:359-375).
    template <typename CallbackOp>
    void ForEach(void* keys, ExtentT keyNum, void* callbackArgs, cudaStream_t stream)
    {
        ForEachAsync<CallbackOp>(keys, keyNum, callbackArgs, stream);
        throw_on(cudaStreamSynchronize(stream) == cudaSuccess ? B2CO_OK : B2CO_ECUDA);
    }
    template <typename CallbackOp>
    void ForEachAsync(void* keys, ExtentT keyNum, void* callbackArgs, cudaStream_t stream)
    {
        detail::for_each_async<CallbackOp, Key, T>(this->handle(), keys, static_cast<SizeType>(keyNum), callbackArgs,
                                                   stream);
    }
#endif

   private:
    Key emptyKey_;
};

// ---- static_set.h ----------------------------------------------------------
template <class Key, class ExtentT = Extent<std::size_t>, class KeyEqual = EqualTo<Key>,
          class ProbingScheme = DoubleHashing<xxhash_32<Key>>, class StorageT = Storage<5>>
class StaticSet : public detail::OpenAddressing<Key, Key, ExtentT, KeyEqual, ProbingScheme, StorageT> {
    static_assert(sizeof(Key) == 2 || sizeof(Key) == 4 || sizeof(Key) == 8, "keys are 2, 4 or 8 bytes");
    using Base = detail::OpenAddressing<Key, Key, ExtentT, KeyEqual, ProbingScheme, StorageT>;

   public:
    using SizeType = typename Base::SizeType;
    using KeyType = Key;
    using ValueType = Key;
    StaticSet(ExtentT capacity, Key emptyKey, KeyEqual const& pred = {}, ProbingScheme const& probing = {},
              StorageT = {}, cudaStream_t stream = nullptr)
        : Base(capacity, emptyKey, emptyKey, emptyKey, 0, pred, probing, stream)
    {}
    void SetErasedKey(Key erasedKey, cudaStream_t s) { this->SetErased(detail::bits_of(erasedKey), s); }
    Key* Data() const { return static_cast<Key*>(Base::Data()); }
#if defined(__CUDACC__)
    // reference: static_set.h ForEach / ForEachAsync (static_set.inl:247-262); the callback gets the key.
    template <typename CallbackOp>
    void ForEach(void* keys, ExtentT keyNum, void* callbackArgs, cudaStream_t stream)
    {
        ForEachAsync<CallbackOp>(keys, keyNum, callbackArgs, stream);
        throw_on(cudaStreamSynchronize(stream) == cudaSuccess ? B2CO_OK : B2CO_ECUDA);
    }
    template <typename CallbackOp>
    void ForEachAsync(void* keys, ExtentT keyNum, void* callbackArgs, cudaStream_t stream)
    {
        detail::for_each_async<CallbackOp, Key, void>(this->handle(), keys, static_cast<SizeType>(keyNum),
                                                      callbackArgs, stream);
    }
#endif
};

// ---- dynamic_map.h ---------------------------------------------------------
template <class Key, class T, class ExtentT = Extent<std::size_t>, class KeyEqual = EqualTo<Key>,
          class ProbingScheme = LinearProbing<murmurhash3_32<Key>>, class StorageT = Storage<5>>
class DynamicMap {
    static_assert(sizeof(Key) == 2 || sizeof(Key) == 4 || sizeof(Key) == 8, "keys are 2, 4 or 8 bytes");
    static_assert(sizeof(Key) == 2 ? sizeof(T) == 2 : (sizeof(T) == 4 || sizeof(T) == 8),
                  "2-byte keys take 2-byte payloads; wider keys take 4- or 8-byte payloads");

   public:
    using SizeType = typename ExtentT::ValueType;
    enum class InsertMode { kExactDedup, kAppendUnique };

    DynamicMap(ExtentT initialCapacity, Key emptyKey, T emptyValue, Key erasedKey, KeyEqual const& pred = {},
               ProbingScheme const& probing = {}, StorageT = {}, cudaStream_t stream = nullptr)
    {
        detail::validate_default(probing, "ProbingScheme");
        detail::validate_default(pred, "KeyEqual");
        b2co_oa_desc d{};
        d.key_bytes = sizeof(Key);
        d.value_bytes = sizeof(T);
        d.bucket_size = StorageT::bucketSize;
        d.probing = ProbingScheme::probing;
        d.hash = ProbingScheme::hash;
        d.key_kind = detail::is_float_key<Key> ? B2CO_KEY_FLOAT : B2CO_KEY_INTEGER;
        d.empty_key_bits = detail::bits_of(emptyKey);
        d.empty_value_bits = detail::bits_of(emptyValue);
        d.erased_key_bits = detail::bits_of(erasedKey);
        throw_on(b2co_dmap_create(&d, static_cast<SizeType>(initialCapacity), to_stream(stream), &m_));
    }
    ~DynamicMap() { b2co_dmap_destroy(m_); }
    DynamicMap(DynamicMap const&) = delete;
    DynamicMap& operator=(DynamicMap const&) = delete;
    DynamicMap(DynamicMap&& o) noexcept : m_{std::exchange(o.m_, nullptr)} {}

    SizeType Size() const { return get(b2co_dmap_size); }
    SizeType Capacity() const { return get(b2co_dmap_capacity); }
    std::size_t NumSubmaps() const { return get(b2co_dmap_num_submaps); }
    void Reserve(SizeType n, cudaStream_t s) { throw_on(b2co_dmap_reserve(m_, n, to_stream(s))); }
    SizeType Insert(void* v, ExtentT n, cudaStream_t s, InsertMode mode = InsertMode::kExactDedup)
    {
        uint64_t r = 0;
        throw_on(b2co_dmap_insert(m_, v, static_cast<SizeType>(n), mode == InsertMode::kAppendUnique, to_stream(s), &r));
        return SizeType(r);
    }
    SizeType InsertOrAssign(void* v, ExtentT n, cudaStream_t s)
    {
        uint64_t r = 0;
        throw_on(b2co_dmap_insert_or_assign(m_, v, static_cast<SizeType>(n), to_stream(s), &r));
        return SizeType(r);
    }
    void Find(void* k, void* o, ExtentT n, cudaStream_t s) { throw_on(b2co_dmap_find(m_, k, o, static_cast<SizeType>(n), to_stream(s))); }
    void Contains(void* k, void* o, ExtentT n, cudaStream_t s)
    {
        throw_on(b2co_dmap_contains(m_, k, static_cast<uint8_t*>(o), static_cast<SizeType>(n), to_stream(s)));
    }
    SizeType Erase(void* k, ExtentT n, cudaStream_t s)
    {
        uint64_t r = 0;
        throw_on(b2co_dmap_erase(m_, k, static_cast<SizeType>(n), to_stream(s), &r));
        return SizeType(r);
    }
    void Clear(cudaStream_t s) { throw_on(b2co_dmap_clear(m_, to_stream(s))); }

   private:
    template <class F>
    SizeType get(F f) const
    {
        uint64_t v = 0;
        throw_on(f(m_, &v));
        return SizeType(v);
    }
    b2co_dmap* m_ = nullptr;
};

// ---- static_multiset.h -----------------------------------------------------
template <class Key>
class StaticMultiset {
    static_assert(std::is_same<Key, int32_t>::value || std::is_same<Key, int64_t>::value,
                  "StaticMultiset supports int32_t and int64_t keys");

   public:
    using Extent = b2co::Extent<std::size_t>;
    using SizeType = std::size_t;
    StaticMultiset(Extent capacity, Key emptyKey, cudaStream_t stream = nullptr)
    {
        throw_on(b2co_mset_create(static_cast<SizeType>(capacity), sizeof(Key), detail::bits_of(emptyKey),
                                  to_stream(stream), &s_));
    }
    ~StaticMultiset() { b2co_mset_destroy(s_); }
    StaticMultiset(StaticMultiset const&) = delete;
    StaticMultiset& operator=(StaticMultiset const&) = delete;
    StaticMultiset(StaticMultiset&& o) noexcept : s_{std::exchange(o.s_, nullptr)} {}
    StaticMultiset& operator=(StaticMultiset&& o) noexcept
    {
        if (this != &o) {
            b2co_mset_destroy(s_);
            s_ = std::exchange(o.s_, nullptr);
        }
        return *this;
    }
    SizeType Capacity() const noexcept
    {
        uint64_t c = 0;
        return b2co_mset_capacity(s_, &c) == B2CO_OK ? SizeType(c) : 0;
    }
    SizeType Size(cudaStream_t = nullptr) const { return get(b2co_mset_size); }
    void Clear(cudaStream_t s = nullptr) { throw_on(b2co_mset_clear(s_, to_stream(s))); }
    SizeType Insert(void* keys, Extent n, cudaStream_t s = nullptr)
    {
        uint64_t f = 0;
        throw_on(b2co_mset_insert(s_, keys, static_cast<SizeType>(n), to_stream(s), &f));
        return SizeType(f);
    }
    template <typename Stencil, typename Predicate = AlwaysTrue>
    SizeType InsertIf(void* keys, Stencil* stencil, Extent n, cudaStream_t s = nullptr)
    {
        static_assert(sizeof(Stencil) == 1, "the C ABI carries uint8 stencils (nonzero = selected)");
        uint64_t f = 0;
        throw_on(b2co_mset_insert_if(s_, keys, reinterpret_cast<uint8_t const*>(stencil), static_cast<SizeType>(n),
                                     to_stream(s), &f));
        return SizeType(f);
    }
    void Contains(void* keys, void* out, Extent n, cudaStream_t s = nullptr)
    {
        throw_on(b2co_mset_contains(s_, keys, static_cast<uint8_t*>(out), static_cast<SizeType>(n), to_stream(s)));
    }
    void Contains(void* keys, Extent n, void* out, cudaStream_t s = nullptr) { Contains(keys, out, n, s); }
    void Find(void* keys, void* out, Extent n, cudaStream_t s = nullptr)
    {
        throw_on(b2co_mset_find(s_, keys, out, static_cast<SizeType>(n), to_stream(s)));
    }
    void Find(void* keys, Extent n, void* out, cudaStream_t s = nullptr) { Find(keys, out, n, s); }
    template <typename Stencil, typename Predicate = AlwaysTrue>
    void ContainsIf(void* keys, Stencil* stencil, void* out, Extent n, cudaStream_t s = nullptr)
    {
        throw_on(b2co_mset_contains_if(s_, keys, reinterpret_cast<uint8_t const*>(stencil), static_cast<uint8_t*>(out),
                                       static_cast<SizeType>(n), to_stream(s)));
    }
    template <typename Stencil, typename Predicate = AlwaysTrue>
    void FindIf(void* keys, Stencil* stencil, void* out, Extent n, cudaStream_t s = nullptr)
    {
        throw_on(b2co_mset_find_if(s_, keys, reinterpret_cast<uint8_t const*>(stencil), out, static_cast<SizeType>(n),
                                   to_stream(s)));
    }
    void CountEach(void* keys, void* out, Extent n, cudaStream_t s = nullptr)
    {
        throw_on(b2co_mset_count_each(s_, keys, static_cast<uint64_t*>(out), static_cast<SizeType>(n), to_stream(s)));
    }
    void CountEachOuter(void* keys, void* out, Extent n, cudaStream_t s = nullptr)
    {
        throw_on(b2co_mset_count_each_outer(s_, keys, static_cast<uint64_t*>(out), static_cast<SizeType>(n),
                                            to_stream(s)));
    }
    SizeType Count(void* keys, Extent n, cudaStream_t s = nullptr)
    {
        uint64_t t = 0;
        throw_on(b2co_mset_count(s_, keys, static_cast<SizeType>(n), to_stream(s), &t));
        return SizeType(t);
    }
    SizeType Retrieve(void* keys, Extent n, void* probeOutput, void* matchOutput, Extent outputCapacity,
                      cudaStream_t s = nullptr)
    {
        uint64_t w = 0;
        throw_on(b2co_mset_retrieve(s_, keys, static_cast<SizeType>(n), probeOutput, matchOutput,
                                    static_cast<SizeType>(outputCapacity), to_stream(s), &w));
        return SizeType(w);
    }
    SizeType RetrieveAll(void* output, Extent outputCapacity, cudaStream_t s = nullptr)
    {
        uint64_t w = 0;
        throw_on(b2co_mset_retrieve_all(s_, output, static_cast<SizeType>(outputCapacity), to_stream(s), &w));
        return SizeType(w);
    }

   private:
    template <class F>
    SizeType get(F f) const
    {
        uint64_t v = 0;
        throw_on(f(s_, &v));
        return SizeType(v);
    }
    b2co_mset* s_ = nullptr;
};

// ---- static_multimap.h -----------------------------------------------------
template <class Key, class Value>
class StaticMultimap {
    static_assert((std::is_same<Key, int32_t>::value || std::is_same<Key, int64_t>::value) &&
                      (std::is_same<Value, int32_t>::value || std::is_same<Value, int64_t>::value),
                  "StaticMultimap supports signed I32/I64 keys and values");

   public:
    using ExtentType = b2co::Extent<std::size_t>;
    using SizeType = std::size_t;
    StaticMultimap(ExtentType capacity, Key emptyKey, Value emptyValue, cudaStream_t stream = nullptr)
    {
        throw_on(b2co_mmap_create(static_cast<SizeType>(capacity), sizeof(Key), sizeof(Value),
                                  detail::bits_of(emptyKey), detail::bits_of(emptyValue), to_stream(stream), &m_));
    }
    ~StaticMultimap() { b2co_mmap_destroy(m_); }
    StaticMultimap(StaticMultimap const&) = delete;
    StaticMultimap& operator=(StaticMultimap const&) = delete;
    StaticMultimap(StaticMultimap&& o) noexcept : m_{std::exchange(o.m_, nullptr)} {}
    StaticMultimap& operator=(StaticMultimap&& o) noexcept
    {
        if (this != &o) {
            b2co_mmap_destroy(m_);
            m_ = std::exchange(o.m_, nullptr);
        }
        return *this;
    }
    SizeType Capacity() const noexcept
    {
        uint64_t c = 0;
        return b2co_mmap_capacity(m_, &c) == B2CO_OK ? SizeType(c) : 0;
    }
    SizeType Size(cudaStream_t = nullptr) const
    {
        uint64_t v = 0;
        throw_on(b2co_mmap_size(m_, &v));
        return SizeType(v);
    }
    void Clear(cudaStream_t s = nullptr) { throw_on(b2co_mmap_clear(m_, to_stream(s))); }
    SizeType Insert(void* pairs, ExtentType n, cudaStream_t s = nullptr)
    {
        uint64_t f = 0;
        throw_on(b2co_mmap_insert(m_, pairs, static_cast<SizeType>(n), to_stream(s), &f));
        return SizeType(f);
    }
    template <class Stencil, class Predicate = AlwaysTrue>
    SizeType InsertIf(void* pairs, Stencil* stencil, ExtentType n, cudaStream_t s = nullptr)
    {
        static_assert(sizeof(Stencil) == 1, "the C ABI carries uint8 stencils (nonzero = selected)");
        uint64_t f = 0;
        throw_on(b2co_mmap_insert_if(m_, pairs, reinterpret_cast<uint8_t const*>(stencil), static_cast<SizeType>(n),
                                     to_stream(s), &f));
        return SizeType(f);
    }
    void Contains(void* keys, void* output, ExtentType n, cudaStream_t s = nullptr) const
    {
        throw_on(b2co_mmap_contains(m_, keys, static_cast<uint8_t*>(output), static_cast<SizeType>(n), to_stream(s)));
    }
    template <class Stencil, class Predicate = AlwaysTrue>
    void ContainsIf(void* keys, Stencil* stencil, void* output, ExtentType n, cudaStream_t s = nullptr) const
    {
        throw_on(b2co_mmap_contains_if(m_, keys, reinterpret_cast<uint8_t const*>(stencil),
                                       static_cast<uint8_t*>(output), static_cast<SizeType>(n), to_stream(s)));
    }
    void Find(void* keys, void* output, ExtentType n, cudaStream_t s = nullptr) const
    {
        throw_on(b2co_mmap_find(m_, keys, output, static_cast<SizeType>(n), to_stream(s)));
    }
    template <class Stencil, class Predicate = AlwaysTrue>
    void FindIf(void* keys, Stencil* stencil, void* output, ExtentType n, cudaStream_t s = nullptr) const
    {
        throw_on(b2co_mmap_find_if(m_, keys, reinterpret_cast<uint8_t const*>(stencil), output,
                                   static_cast<SizeType>(n), to_stream(s)));
    }
    uint64_t Count(void* keys, ExtentType n, cudaStream_t s = nullptr) const
    {
        uint64_t t = 0;
        throw_on(b2co_mmap_count(m_, keys, static_cast<SizeType>(n), to_stream(s), &t));
        return t;
    }
    SizeType Retrieve(void* keys, ExtentType n, void* probeOut, void* valueOut, ExtentType outputCapacity,
                      cudaStream_t s = nullptr) const
    {
        uint64_t w = 0;
        throw_on(b2co_mmap_retrieve(m_, keys, static_cast<SizeType>(n), probeOut, valueOut,
                                    static_cast<SizeType>(outputCapacity), to_stream(s), &w));
        return SizeType(w);
    }
    SizeType RetrieveAll(void* keyOut, void* valueOut, ExtentType outputCapacity, cudaStream_t s = nullptr) const
    {
        uint64_t w = 0;
        throw_on(b2co_mmap_retrieve_all(m_, keyOut, valueOut, static_cast<SizeType>(outputCapacity), to_stream(s),
                                        &w));
        return SizeType(w);
    }

   private:
    b2co_mmap* m_ = nullptr;
};

// ---- roaring_bitmap.h ------------------------------------------------------
template <typename Key, typename ExtentT = Extent<std::size_t>>
class RoaringBitmap {
    static_assert(std::is_same<Key, uint32_t>::value || std::is_same<Key, uint64_t>::value,
                  "RoaringBitmap key type must be uint32_t or uint64_t");

   public:
    using KeyType = Key;
    using SizeType = typename ExtentT::ValueType;
    // A complete, trusted serialized bitmap in host memory (length from the format).
    explicit RoaringBitmap(void const* bitmap, cudaStream_t stream = nullptr) : RoaringBitmap(bitmap, ~std::size_t(0), stream) {}
    // A serialized bitmap of at most bitmapBytes bytes; the parse is bounds-checked.
    RoaringBitmap(void const* bitmap, std::size_t bitmapBytes, cudaStream_t stream = nullptr)
    {
        throw_on(b2co_roaring_create(bitmap, bitmapBytes, sizeof(Key), to_stream(stream), &r_));
    }
    ~RoaringBitmap() { b2co_roaring_destroy(r_); }
    RoaringBitmap(RoaringBitmap const&) = delete;
    RoaringBitmap& operator=(RoaringBitmap const&) = delete;
    RoaringBitmap(RoaringBitmap&& o) noexcept : r_{std::exchange(o.r_, nullptr)} {}
    RoaringBitmap& operator=(RoaringBitmap&& o) noexcept
    {
        if (this != &o) {
            b2co_roaring_destroy(r_);
            r_ = std::exchange(o.r_, nullptr);
        }
        return *this;
    }
    void Contains(void const* keys, void* outputValues, ExtentT keyNum, cudaStream_t stream) const
    {
        throw_on(b2co_roaring_contains(r_, keys, static_cast<uint8_t*>(outputValues), static_cast<SizeType>(keyNum),
                                       to_stream(stream)));
    }
    void ContainsAsync(void const* keys, void* outputValues, ExtentT keyNum, cudaStream_t stream) const
    {
        throw_on(b2co_roaring_contains_async(r_, keys, static_cast<uint8_t*>(outputValues),
                                             static_cast<SizeType>(keyNum), to_stream(stream)));
    }
    uint64_t Size() const noexcept
    {
        uint64_t v = 0;
        return b2co_roaring_size(r_, &v) == B2CO_OK ? v : 0;
    }
    bool Empty() const noexcept { return Size() == 0; }
    uint64_t SizeBytes() const noexcept
    {
        uint64_t v = 0;
        return b2co_roaring_size_bytes(r_, &v) == B2CO_OK ? v : 0;
    }
    uint8_t const* Data() const noexcept
    {
        uint8_t const* p = nullptr;
        return b2co_roaring_data(r_, &p) == B2CO_OK ? p : nullptr;
    }

   private:
    b2co_roaring* r_ = nullptr;
};

// ---- bloom_filter.h --------------------------------------------------------
// The reference's template parameters, in its order (bloom_filter_policy.h:42-48).
// WordsPerBlock and PatternBits select the bits; the layout and
// ConditionalAdd / EarlyExitContains parameters only steer the reference's work
// distribution and are accepted for source compatibility.
template <class Key, class Hash = xxhash_64<Key>, class Word = uint32_t, uint32_t WordsPerBlock = 32 / sizeof(Word),
          uint32_t PatternBits = WordsPerBlock, uint32_t AddHorizontalLayout = WordsPerBlock,
          uint32_t AddVerticalLayout = 1, uint32_t ContainsHorizontalLayout = 1,
          uint32_t ContainsVerticalLayout = WordsPerBlock, bool ConditionalAdd = false, bool EarlyExitContains = false>
struct BloomFilterPolicy {
    static_assert(std::is_same<Word, uint32_t>::value, "BloomFilter currently supports uint32_t words only");
    static_assert(WordsPerBlock != 0 && (WordsPerBlock & (WordsPerBlock - 1)) == 0 && WordsPerBlock <= 32,
                  "WordsPerBlock must be a non-zero power of two not above 32");
    static_assert(PatternBits >= WordsPerBlock && PatternBits <= 64 && PatternBits <= 32 * WordsPerBlock &&
                      PatternBits % WordsPerBlock == 0,
                  "PatternBits must be evenly distributed across the words and fit the salt table");
    static_assert(WordsPerBlock % (AddHorizontalLayout * AddVerticalLayout) == 0 &&
                      WordsPerBlock % (ContainsHorizontalLayout * ContainsVerticalLayout) == 0,
                  "layouts must evenly divide WordsPerBlock");
    using KeyType = Key;
    using Hasher = Hash;
    using WordType = Word;
    static constexpr uint32_t wordsPerBlock = WordsPerBlock;
    static constexpr uint32_t patternBits = PatternBits;
    constexpr BloomFilterPolicy(Hash h = {}) : seed_{h.seed_} {}
    constexpr bool operator==(BloomFilterPolicy const& o) const { return seed_ == o.seed_; }
    uint64_t seed_;
};

template <class Hash, class Word, uint32_t WordsPerBlock>
using DefaultFilterPolicy = BloomFilterPolicy<typename Hash::ArgumentType, Hash, Word, WordsPerBlock>;

template <class Key>
using ArrowFilterPolicy = BloomFilterPolicy<Key, xxhash_64<Key>, uint32_t, 8, 8, 8, 1, 1, 8, false, false>;

template <class Key, class ExtentT = Extent<std::size_t>, class Policy = BloomFilterPolicy<Key>>
class BloomFilter {
    static_assert(sizeof(Key) == 4 || sizeof(Key) == 8, "BloomFilter supports 4- and 8-byte keys");

   public:
    using SizeType = typename ExtentT::ValueType;
    using WordType = uint32_t;
    explicit BloomFilter(ExtentT numBlocks, Policy const& policy = Policy{}, cudaStream_t stream = nullptr)
    {
        throw_on(b2co_bloom_create_policy(static_cast<SizeType>(numBlocks), sizeof(Key), policy.seed_,
                                          Policy::wordsPerBlock, Policy::patternBits, to_stream(stream), &f_));
    }
    ~BloomFilter() { b2co_bloom_destroy(f_); }
    BloomFilter(BloomFilter const&) = delete;
    BloomFilter& operator=(BloomFilter const&) = delete;
    BloomFilter(BloomFilter&& o) noexcept : f_{std::exchange(o.f_, nullptr)} {}

    void Clear(cudaStream_t s = nullptr) { throw_on(b2co_bloom_clear(f_, to_stream(s))); }
    void ClearAsync(cudaStream_t s = nullptr) { throw_on(b2co_bloom_clear_async(f_, to_stream(s))); }
    void Add(void* k, ExtentT n, cudaStream_t s = nullptr) { throw_on(b2co_bloom_add(f_, k, static_cast<SizeType>(n), to_stream(s))); }
    void AddAsync(void* k, ExtentT n, cudaStream_t s = nullptr) { throw_on(b2co_bloom_add_async(f_, k, static_cast<SizeType>(n), to_stream(s))); }
    void AddIf(void* k, void* st, ExtentT n, cudaStream_t s = nullptr)
    {
        throw_on(b2co_bloom_add_if(f_, k, static_cast<uint8_t const*>(st), static_cast<SizeType>(n), to_stream(s)));
    }
    void Contains(void* k, ExtentT n, void* o, cudaStream_t s = nullptr) const
    {
        throw_on(b2co_bloom_contains(f_, k, static_cast<uint8_t*>(o), static_cast<SizeType>(n), to_stream(s)));
    }
    void ContainsAsync(void* k, ExtentT n, void* o, cudaStream_t s = nullptr) const
    {
        throw_on(b2co_bloom_contains_async(f_, k, static_cast<uint8_t*>(o), static_cast<SizeType>(n), to_stream(s)));
    }
    void ContainsIf(void* k, void* st, void* o, ExtentT n, cudaStream_t s = nullptr) const
    {
        throw_on(b2co_bloom_contains_if(f_, k, static_cast<uint8_t const*>(st), static_cast<uint8_t*>(o), static_cast<SizeType>(n), to_stream(s)));
    }
    void Merge(BloomFilter const& o, cudaStream_t s = nullptr) { throw_on(b2co_bloom_merge(f_, o.f_, to_stream(s))); }
    void MergeAsync(BloomFilter const& o, cudaStream_t s = nullptr) { throw_on(b2co_bloom_merge_async(f_, o.f_, to_stream(s))); }
    void Intersect(BloomFilter const& o, cudaStream_t s = nullptr) { throw_on(b2co_bloom_intersect(f_, o.f_, to_stream(s))); }
    void IntersectAsync(BloomFilter const& o, cudaStream_t s = nullptr) { throw_on(b2co_bloom_intersect_async(f_, o.f_, to_stream(s))); }
    WordType* Data()
    {
        uint32_t* w = nullptr;
        throw_on(b2co_bloom_data(f_, &w));
        return w;
    }
    ExtentT BlockExtent() const
    {
        uint64_t n = 0;
        throw_on(b2co_bloom_num_blocks(f_, &n));
        return ExtentT(SizeType(n));
    }
    SizeType NumWords() const { return SizeType(static_cast<SizeType>(BlockExtent()) * Policy::wordsPerBlock); }
    std::size_t SizeBytes() const { return std::size_t(NumWords()) * sizeof(WordType); }

   private:
    b2co_bloom* f_ = nullptr;
};

// ---- hyperloglog.h ---------------------------------------------------------
template <class Key>
class HyperLogLog {
    static_assert(std::is_same_v<Key, int32_t> || std::is_same_v<Key, int64_t>, "HyperLogLog supports int32_t and int64_t");

   public:
    using ExtentType = Extent<std::size_t>;
    static HyperLogLog CreateWithSketchSizeKB(uint32_t kb, cudaStream_t s = nullptr)
    {
        uint32_t p = 0;
        throw_on(b2co_hll_precision_for_sketch_kb(kb, &p));
        return HyperLogLog(p, s);
    }
    static HyperLogLog CreateWithStandardDeviation(double d, cudaStream_t s = nullptr)
    {
        uint32_t p = 0;
        throw_on(b2co_hll_precision_for_deviation(d, &p));
        return HyperLogLog(p, s);
    }
    static HyperLogLog CreateWithPrecision(uint32_t p, cudaStream_t s = nullptr) { return HyperLogLog(p, s); }
    HyperLogLog(HyperLogLog const&) = delete;
    HyperLogLog& operator=(HyperLogLog const&) = delete;
    HyperLogLog(HyperLogLog&& o) noexcept : h_{std::exchange(o.h_, nullptr)}, p_{o.p_} {}
    ~HyperLogLog() { b2co_hll_destroy(h_); }

    uint32_t SketchSizeKB() const noexcept { return h_ ? (1u << p_) / 1024u : 0u; }
    void Clear(cudaStream_t s = nullptr) { throw_on(b2co_hll_clear(h_, to_stream(s))); }
    void Add(void* k, ExtentType n, cudaStream_t s = nullptr) { throw_on(b2co_hll_add(h_, k, static_cast<std::size_t>(n), to_stream(s))); }
    void Merge(HyperLogLog const& o, cudaStream_t s = nullptr) { throw_on(b2co_hll_merge(h_, o.h_, to_stream(s))); }
    uint64_t Estimate(cudaStream_t s = nullptr) const
    {
        uint64_t e = 0;
        throw_on(b2co_hll_estimate(h_, to_stream(s), &e));
        return e;
    }
    uint8_t const* Data() const noexcept
    {
        uint8_t const* r = nullptr;
        return b2co_hll_data(h_, &r) == B2CO_OK ? r : nullptr;
    }

   private:
    HyperLogLog(uint32_t p, cudaStream_t s) : p_{p} { throw_on(b2co_hll_create(p, sizeof(Key), to_stream(s), &h_)); }
    b2co_hll* h_ = nullptr;
    uint32_t p_ = 0;
};

}  // namespace b2co

#if defined(__CUDACC__)
#include "for_each.cuh"
#endif
