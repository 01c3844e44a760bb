// ForEach with caller-defined device functors, compiled by nvcc the way a user
// of the C++ API compiles it: the counting functors of the reference's
// tests/static_map/for_each_test.cpp and tests/static_set/for_each_test.cpp,
// over inserted keys, absent keys and the empty key, for LinearProbing and
// DoubleHashing, bucket sizes 1 and 5, 4- and 8-byte keys.  Expected counts
// come from the host.  Built and run by tests/test_for_each_gpu.py.
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "b2co/b2co.hpp"

#define CHECK(cond)                                                                      \
    do {                                                                                 \
        if (!(cond)) {                                                                   \
            std::fprintf(stderr, "CHECK failed %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            std::exit(1);                                                                \
        }                                                                                \
    } while (0)

namespace {

template <class Key, class Value>
struct CountEvenKeyWithValueOne {
    unsigned int* counter;
    __device__ CountEvenKeyWithValueOne(uint8_t* state) : counter{reinterpret_cast<unsigned int*>(state)} {}
    template <class K, class V>
    __device__ void operator()(b2co::Pair<K, V> slot) const
    {
        if (slot.first % 2 == 0 && slot.second == 1) atomicAdd(counter, 1u);
    }
};

template <class Key, class Value>
struct CountAllPairs {
    unsigned int* counter;
    __device__ CountAllPairs(uint8_t* state) : counter{reinterpret_cast<unsigned int*>(state)} {}
    template <class K, class V>
    __device__ void operator()(b2co::Pair<K, V>) const
    {
        atomicAdd(counter, 1u);
    }
};

template <class Key>
struct CountEvenKeys {
    unsigned int* counter;
    __device__ CountEvenKeys(uint8_t* state) : counter{reinterpret_cast<unsigned int*>(state)} {}
    __device__ void operator()(Key k) const
    {
        if (k % 2 == 0) atomicAdd(counter, 1u);
    }
};

template <class Key>
struct CountAllKeys {
    unsigned int* counter;
    __device__ CountAllKeys(uint8_t* state) : counter{reinterpret_cast<unsigned int*>(state)} {}
    __device__ void operator()(Key) const { atomicAdd(counter, 1u); }
};

template <class T>
T* upload(std::vector<T> const& h)
{
    T* d = nullptr;
    CHECK(cudaMalloc(reinterpret_cast<void**>(&d), sizeof(T) * (h.size() ? h.size() : 1)) == cudaSuccess);
    if (!h.empty()) CHECK(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess);
    return d;
}

unsigned int read_counter(unsigned int* d)
{
    unsigned int h = 0;
    CHECK(cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost) == cudaSuccess);
    return h;
}

// Inserted keys 1..n spread by an odd multiplier; values 1 for every third key.
template <class Key>
std::vector<Key> inserted_keys(size_t n)
{
    std::vector<Key> k(n);
    for (size_t i = 0; i < n; ++i) k[i] = Key((i + 1) * 2654435761ull % (Key(1) << (sizeof(Key) * 8 - 2)));
    return k;
}

template <class Key, class Value, class Probe, int B>
void map_case()
{
    cudaStream_t s;
    CHECK(cudaStreamCreate(&s) == cudaSuccess);
    size_t const n = 20000;
    using Map = b2co::StaticMap<Key, Value, b2co::Extent<size_t>, b2co::EqualTo<Key>, Probe, b2co::Storage<B>>;
    Key const empty = Key(~Key(0));
    Map map(b2co::Extent<size_t>{2 * n}, empty, Value(~Value(0)), {}, {}, {}, s);
    auto keys = inserted_keys<Key>(n);
    std::vector<b2co::Pair<Key, Value>> pairs(n);
    unsigned int expect_even_one = 0;
    for (size_t i = 0; i < n; ++i) {
        pairs[i] = {keys[i], Value(i % 3 == 0 ? 1 : 2)};
        expect_even_one += (keys[i] % 2 == 0 && i % 3 == 0);
    }
    auto* dp = upload(pairs);
    CHECK(map.Insert(dp, n, s) == 0);
    // probe keys: every inserted key, as many absent ones, and the empty key
    std::vector<Key> probe(keys);
    for (size_t i = 0; i < n; ++i) probe.push_back(Key((Key(1) << (sizeof(Key) * 8 - 2)) + Key(i)));
    probe.push_back(empty);
    auto* dk = upload(probe);
    unsigned int* counter = nullptr;
    CHECK(cudaMalloc(reinterpret_cast<void**>(&counter), sizeof(unsigned int)) == cudaSuccess);

    CHECK(cudaMemset(counter, 0, sizeof(unsigned int)) == cudaSuccess);
    map.template ForEach<CountEvenKeyWithValueOne<Key, Value>>(dk, probe.size(), counter, s);
    CHECK(read_counter(counter) == expect_even_one);

    CHECK(cudaMemset(counter, 0, sizeof(unsigned int)) == cudaSuccess);
    map.template ForEachAsync<CountAllPairs<Key, Value>>(dk, probe.size(), counter, s);
    CHECK(cudaStreamSynchronize(s) == cudaSuccess);
    CHECK(read_counter(counter) == n);

    // zero keys and a null key array are no-ops; an oversized batch is a length error
    CHECK(cudaMemset(counter, 0, sizeof(unsigned int)) == cudaSuccess);
    map.template ForEach<CountAllPairs<Key, Value>>(dk, 0, counter, s);
    map.template ForEach<CountAllPairs<Key, Value>>(nullptr, probe.size(), counter, s);
    CHECK(read_counter(counter) == 0);
    bool threw = false;
    try {
        map.template ForEachAsync<CountAllPairs<Key, Value>>(dk, size_t(1) << 32, counter, s);
    } catch (std::length_error const&) {
        threw = true;
    }
    CHECK(threw);
    cudaFree(counter);
    cudaFree(dk);
    cudaFree(dp);
    cudaStreamDestroy(s);
}

template <class Key, class Probe, int B>
void set_case()
{
    cudaStream_t s;
    CHECK(cudaStreamCreate(&s) == cudaSuccess);
    size_t const n = 15000;
    using Set = b2co::StaticSet<Key, b2co::Extent<size_t>, b2co::EqualTo<Key>, Probe, b2co::Storage<B>>;
    Key const empty = Key(~Key(0));
    Set set(b2co::Extent<size_t>{2 * n}, empty, {}, {}, {}, s);
    auto keys = inserted_keys<Key>(n);
    unsigned int expect_even = 0;
    for (auto k : keys) expect_even += (k % 2 == 0);
    auto* dkeys = upload(keys);
    CHECK(set.Insert(dkeys, n, s) == 0);
    std::vector<Key> probe(keys);
    for (size_t i = 0; i < n; ++i) probe.push_back(Key((Key(1) << (sizeof(Key) * 8 - 2)) + Key(i)));
    probe.push_back(empty);
    auto* dk = upload(probe);
    unsigned int* counter = nullptr;
    CHECK(cudaMalloc(reinterpret_cast<void**>(&counter), sizeof(unsigned int)) == cudaSuccess);
    CHECK(cudaMemset(counter, 0, sizeof(unsigned int)) == cudaSuccess);
    set.template ForEach<CountEvenKeys<Key>>(dk, probe.size(), counter, s);
    CHECK(read_counter(counter) == expect_even);
    CHECK(cudaMemset(counter, 0, sizeof(unsigned int)) == cudaSuccess);
    set.template ForEach<CountAllKeys<Key>>(dk, probe.size(), counter, s);
    CHECK(read_counter(counter) == n);
    cudaFree(counter);
    cudaFree(dk);
    cudaFree(dkeys);
    cudaStreamDestroy(s);
}

}  // namespace

int main()
{
    using namespace b2co;
    map_case<uint32_t, uint32_t, LinearProbing<murmurhash3_32<uint32_t>>, 1>();
    map_case<uint32_t, uint32_t, LinearProbing<murmurhash3_32<uint32_t>>, 5>();
    map_case<uint32_t, uint32_t, DoubleHashing<xxhash_32<uint32_t>>, 5>();
    map_case<uint64_t, uint64_t, LinearProbing<murmurhash3_32<uint64_t>>, 1>();
    map_case<uint64_t, uint64_t, LinearProbing<murmurhash3_32<uint64_t>>, 5>();
    map_case<uint64_t, uint64_t, DoubleHashing<xxhash_32<uint64_t>>, 5>();
    map_case<int64_t, int32_t, DoubleHashing<xxhash_32<int64_t>>, 5>();
    set_case<uint32_t, DoubleHashing<xxhash_32<uint32_t>>, 5>();
    set_case<uint64_t, LinearProbing<murmurhash3_32<uint64_t>>, 1>();
    std::printf("for_each test ok\n");
    return 0;
}
