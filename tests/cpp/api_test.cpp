// C++ API test: the reference's class templates, used the way its own tests use
// them (tests/static_map/find_test.cpp, insert_test.cpp, static_set/*,
// dynamic_map/*, bloom_filter/*, hyperloglog/*), against std::unordered_map /
// std::unordered_set goldens (tests/common/golden.h).  Built and run by
// tests/test_cpp_api_gpu.py.
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <random>
#include <stdexcept>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <cuda_runtime_api.h>

#include "b2co/b2co.hpp"

#define CHECK(cond)                                                              \
    do {                                                                         \
        if (!(cond)) {                                                           \
            std::fprintf(stderr, "CHECK failed %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            std::exit(1);                                                        \
        }                                                                        \
    } while (0)

template <class T>
struct DeviceBuffer {
    T* p = nullptr;
    size_t n = 0;
    explicit DeviceBuffer(size_t count) : n(count)
    {
        CHECK(cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (count ? count : 1)) == cudaSuccess);
    }
    DeviceBuffer(std::vector<T> const& h) : DeviceBuffer(h.size()) { upload(h); }
    ~DeviceBuffer() { cudaFree(p); }
    void upload(std::vector<T> const& h) { CHECK(cudaMemcpy(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess); }
    std::vector<T> download() const
    {
        std::vector<T> h(n);
        CHECK(cudaMemcpy(h.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost) == cudaSuccess);
        return h;
    }
};

template <class E, class F>
void expect_throw(F f)
{
    try {
        f();
    } catch (E const&) {
        return;
    }
    std::fprintf(stderr, "expected exception not thrown\n");
    std::exit(1);
}

int main()
{
    cudaStream_t stream;
    CHECK(cudaStreamCreate(&stream) == cudaSuccess);
    std::mt19937_64 gen(200);

    // ---- StaticMap<int64_t,int64_t>, DoubleHashing<xxhash_32>, Storage<5> ----
    {
        using Map = b2co::StaticMap<int64_t, int64_t, b2co::Extent<size_t>, b2co::EqualTo<int64_t>,
                                    b2co::DoubleHashing<b2co::xxhash_32<int64_t>>, b2co::Storage<5>>;
        const size_t n = 200000;
        Map map(b2co::Extent<size_t>{2 * n}, -1, -1, {}, {}, {}, stream);
        std::unordered_map<int64_t, int64_t> golden;
        std::vector<b2co::Pair<int64_t, int64_t>> pairs;
        std::uniform_int_distribution<int64_t> dist(1, 2 * int64_t(n));
        while (pairs.size() < n) {
            int64_t k = dist(gen);
            if (golden.emplace(k, 3 * k + 1).second) pairs.push_back({k, 3 * k + 1});
        }
        DeviceBuffer<b2co::Pair<int64_t, int64_t>> dpairs(pairs);
        CHECK(map.Insert(dpairs.p, b2co::Extent<size_t>{n}, stream) == 0);
        CHECK(map.Insert(dpairs.p, b2co::Extent<size_t>{1000}, stream) == 1000);  // duplicates fail
        std::vector<int64_t> q(2 * n);
        for (auto& x : q) x = dist(gen);
        DeviceBuffer<int64_t> dq(q), dout(q.size());
        DeviceBuffer<uint8_t> dc(q.size());
        map.Find(dq.p, dout.p, b2co::Extent<size_t>{q.size()}, stream);
        map.Contains(dq.p, dc.p, b2co::Extent<size_t>{q.size()}, stream);
        auto out = dout.download();
        auto c = dc.download();
        size_t hits = 0;
        for (size_t i = 0; i < q.size(); ++i) {
            auto it = golden.find(q[i]);
            CHECK(out[i] == (it == golden.end() ? -1 : it->second));
            CHECK(c[i] == (it != golden.end()));
            hits += it != golden.end();
        }
        CHECK(map.Count(dq.p, b2co::Extent<size_t>{q.size()}, stream) == hits);
        // InsertOrAssign: existing keys are assigned, new ones inserted
        std::vector<b2co::Pair<int64_t, int64_t>> upd = {{pairs[0].first, 7}, {int64_t(10 * n), 8}};
        DeviceBuffer<b2co::Pair<int64_t, int64_t>> dupd(upd);
        size_t assigned = 0;
        CHECK(map.InsertOrAssign(dupd.p, b2co::Extent<size_t>{2}, stream, assigned) == 0);
        CHECK(assigned == 1);
        // a probing scheme with instance state cannot reach the device
        expect_throw<std::invalid_argument>([&] {
            Map bad(b2co::Extent<size_t>{100}, -1, -1, {}, b2co::DoubleHashing<b2co::xxhash_32<int64_t>>{5}, {}, stream);
        });
        expect_throw<std::length_error>([&] { map.FindAsync(dq.p, dout.p, b2co::Extent<size_t>{size_t(1) << 32}, stream); });
    }

    // ---- StaticSet<int32_t> (defaults: DoubleHashing<xxhash_32>, Storage<5>) ----
    {
        b2co::StaticSet<int32_t> set(b2co::Extent<size_t>{50000}, -1, {}, {}, {}, stream);
        std::unordered_set<int32_t> golden;
        std::vector<int32_t> keys;
        std::uniform_int_distribution<int32_t> dist(0, 100000);
        for (int i = 0; i < 30000; ++i) {
            int32_t k = dist(gen);
            keys.push_back(k);
            golden.insert(k);
        }
        DeviceBuffer<int32_t> dk(keys);
        CHECK(set.Insert(dk.p, b2co::Extent<size_t>{keys.size()}, stream) == keys.size() - golden.size());
        DeviceBuffer<int32_t> out(keys.size());
        set.Find(dk.p, out.p, b2co::Extent<size_t>{keys.size()}, stream);
        auto o = out.download();
        for (size_t i = 0; i < keys.size(); ++i) CHECK(o[i] == keys[i]);
    }

    // ---- DynamicMap<int32_t,int32_t> grows past its initial capacity ----
    {
        b2co::DynamicMap<int32_t, int32_t> dm(b2co::Extent<size_t>{30000}, -1, -1, -2, {}, {}, {}, stream);
        std::vector<b2co::Pair<int32_t, int32_t>> pairs;
        for (int32_t k = 0; k < 100000; ++k) pairs.push_back({k, k ^ 0x5a5a});
        DeviceBuffer<b2co::Pair<int32_t, int32_t>> dp(pairs);
        CHECK(dm.Insert(dp.p, b2co::Extent<size_t>{pairs.size()}, stream) == pairs.size());
        CHECK(dm.Size() == pairs.size());
        std::vector<int32_t> q = {0, 5, 99999, 100000, -7};
        DeviceBuffer<int32_t> dq(q), dout(q.size());
        dm.Find(dq.p, dout.p, b2co::Extent<size_t>{q.size()}, stream);
        auto o = dout.download();
        CHECK(o[0] == (0 ^ 0x5a5a) && o[1] == (5 ^ 0x5a5a) && o[2] == (99999 ^ 0x5a5a) && o[3] == -1 && o[4] == -1);
        expect_throw<std::invalid_argument>([&] {
            b2co::DynamicMap<int32_t, int32_t> bad(b2co::Extent<size_t>{100}, -1, -1, -1, {}, {}, {}, stream);
        });
    }

    // ---- DynamicMap<float,float> and <uint16_t,uint16_t> (dynamic_map tests' key types) ----
    {
        b2co::DynamicMap<float, float> fm(b2co::Extent<size_t>{20000}, -1.0f, -1.0f, -2.0f, {}, {}, {}, stream);
        std::vector<b2co::Pair<float, float>> pairs;
        for (int k = 1; k <= 50000; ++k) pairs.push_back({float(k) * 0.5f, float(k)});
        DeviceBuffer<b2co::Pair<float, float>> dp(pairs);
        CHECK(fm.Insert(dp.p, b2co::Extent<size_t>{pairs.size()}, stream) == pairs.size());
        std::vector<float> q = {0.5f, 100.0f, 0.25f};
        DeviceBuffer<float> dq(q), dout(q.size());
        fm.Find(dq.p, dout.p, b2co::Extent<size_t>{q.size()}, stream);
        auto o = dout.download();
        CHECK(o[0] == 1.0f && o[1] == 200.0f && o[2] == -1.0f);

        b2co::DynamicMap<uint16_t, uint16_t> sm(b2co::Extent<size_t>{4000}, 0xffff, 0, 0xfffe, {}, {}, {}, stream);
        std::vector<b2co::Pair<uint16_t, uint16_t>> sp;
        for (uint16_t k = 0; k < 30000; ++k) sp.push_back({k, uint16_t(k + 1)});
        DeviceBuffer<b2co::Pair<uint16_t, uint16_t>> dsp(sp);
        CHECK(sm.Insert(dsp.p, b2co::Extent<size_t>{sp.size()}, stream) == sp.size());
        std::vector<uint16_t> sq = {0, 29999, 30000};
        DeviceBuffer<uint16_t> dsq(sq), dso(sq.size());
        sm.Find(dsq.p, dso.p, b2co::Extent<size_t>{sq.size()}, stream);
        auto so = dso.download();
        CHECK(so[0] == 1 && so[1] == 30000 && so[2] == 0);
    }

    // ---- BloomFilter<uint64_t>: no false negatives; incompatible merge throws ----
    {
        b2co::BloomFilter<uint64_t> f(b2co::Extent<size_t>{1 << 14}, {}, stream);
        std::vector<uint64_t> keys(100000);
        for (auto& k : keys) k = gen();
        DeviceBuffer<uint64_t> dk(keys);
        DeviceBuffer<uint8_t> out(keys.size());
        f.Add(dk.p, b2co::Extent<size_t>{keys.size()}, stream);
        f.Contains(dk.p, b2co::Extent<size_t>{keys.size()}, out.p, stream);
        for (auto v : out.download()) CHECK(v == 1);
        b2co::BloomFilter<uint64_t> other(b2co::Extent<size_t>{1 << 13}, {}, stream);
        expect_throw<std::invalid_argument>([&] { f.Merge(other, stream); });
        expect_throw<std::length_error>([&] { b2co::BloomFilter<uint64_t> big(b2co::Extent<size_t>{size_t(1) << 32}); });
    }

    // ---- policy aliases (bloom_filter_policy.h:205-211, generalization_test.cpp:32-41) ----
    {
        static_assert(std::is_same<b2co::ArrowFilterPolicy<uint32_t>,
                                   b2co::BloomFilterPolicy<uint32_t, b2co::xxhash_64<uint32_t>, uint32_t, 8, 8, 8, 1,
                                                           1, 8, false, false>>::value,
                      "ArrowFilterPolicy is the 8-word, 8-bit policy");
        using P16 = b2co::DefaultFilterPolicy<b2co::xxhash_64<uint64_t>, uint32_t, 16>;
        static_assert(P16::wordsPerBlock == 16 && P16::patternBits == 16, "DefaultFilterPolicy<..., 16>");
        b2co::BloomFilter<uint64_t, b2co::Extent<size_t>, P16> f(b2co::Extent<size_t>{4096}, P16{}, stream);
        CHECK(f.NumWords() == 4096 * 16);
        std::vector<uint64_t> keys(50000);
        for (auto& k : keys) k = gen();
        DeviceBuffer<uint64_t> dk(keys);
        DeviceBuffer<uint8_t> out(keys.size());
        f.Add(dk.p, b2co::Extent<size_t>{keys.size()}, stream);
        f.Contains(dk.p, b2co::Extent<size_t>{keys.size()}, out.p, stream);
        for (auto v : out.download()) CHECK(v == 1);
        using Seeded = b2co::BloomFilterPolicy<uint32_t, b2co::xxhash_64<uint32_t>, uint32_t, 8, 16, 1, 8, 1, 8, true, true>;
        b2co::BloomFilter<uint32_t, b2co::Extent<size_t>, Seeded> g(b2co::Extent<size_t>{257}, Seeded{b2co::xxhash_64<uint32_t>{42}}, stream);
        CHECK(g.NumWords() == 257 * 8);
    }

    // ---- StaticMultimap / StaticMultiset (contract_test.cpp:18-53, semantics_test.cpp) ----
    {
        using T = int64_t;
        T const lo = std::numeric_limits<T>::lowest();
        b2co::StaticMultimap<T, T> mm(b2co::Extent<size_t>{7}, lo, lo, stream);
        std::vector<b2co::Pair<T, T>> pairs{{-7, 4}, {3, -8}, {3, -8}, {-7, -3}, {9, 7}, {3, 2}, {3, 9}};
        DeviceBuffer<b2co::Pair<T, T>> dp(pairs);
        CHECK(mm.Insert(dp.p, b2co::Extent<size_t>{pairs.size()}, stream) == 0);
        DeviceBuffer<T> q(std::vector<T>{3, -7, 3, 42, lo});
        DeviceBuffer<T> found(5);
        mm.Find(q.p, found.p, b2co::Extent<size_t>{5}, stream);
        CHECK((found.download() == std::vector<T>{-8, -3, -8, lo, lo}));
        CHECK(mm.Count(q.p, b2co::Extent<size_t>{5}, stream) == 10);
        DeviceBuffer<T> ok(10), ov(10);
        CHECK(mm.Retrieve(q.p, b2co::Extent<size_t>{5}, ok.p, ov.p, b2co::Extent<size_t>{10}, stream) == 10);
        CHECK((ov.download() == std::vector<T>{-8, -8, 2, 9, -3, 4, -8, -8, 2, 9}));
        expect_throw<std::length_error>([&] { mm.Retrieve(q.p, b2co::Extent<size_t>{5}, ok.p, ov.p, b2co::Extent<size_t>{9}, stream); });
        expect_throw<std::overflow_error>([&] { mm.Count(q.p, b2co::Extent<size_t>{std::numeric_limits<size_t>::max()}, stream); });
        b2co::StaticMultiset<T> ms(b2co::Extent<size_t>{5}, lo, stream);
        DeviceBuffer<T> keys(std::vector<T>{7, 2, 7, std::numeric_limits<T>::max(), -4, 2, 9});
        CHECK(ms.Insert(keys.p, b2co::Extent<size_t>{7}, stream) == 2);
        CHECK(ms.Size(stream) == 5);
        DeviceBuffer<uint64_t> counts(7);
        ms.CountEach(keys.p, counts.p, b2co::Extent<size_t>{7}, stream);
        CHECK((counts.download() == std::vector<uint64_t>{2, 1, 2, 1, 1, 1, 0}));
        auto moved = std::move(ms);
        CHECK(moved.Size(stream) == 5);
        expect_throw<std::logic_error>([&] { ms.Clear(stream); });
    }

    // ---- RoaringBitmap<uint32_t>: the three-key portable bitmap (roaring_bitmap_factory.h AcceptanceKeys) ----
    {
        // cookie 12346, one container: key 1, cardinality 3 (stored as 2), offset 16, values 2, 4, 8
        std::vector<uint8_t> bytes{0x3a, 0x30, 0, 0, 1, 0, 0, 0, 1, 0, 2, 0, 16, 0, 0, 0, 2, 0, 4, 0, 8, 0};
        b2co::RoaringBitmap<uint32_t> rb(bytes.data(), bytes.size(), stream);
        CHECK(rb.Size() == 3 && rb.SizeBytes() == bytes.size() && !rb.Empty());
        DeviceBuffer<uint32_t> q(std::vector<uint32_t>{(1u << 16) | 2u, (1u << 16) | 3u, (1u << 16) | 8u, 2u});
        DeviceBuffer<uint8_t> out(4);
        rb.Contains(q.p, out.p, b2co::Extent<size_t>{4}, stream);
        CHECK((out.download() == std::vector<uint8_t>{1, 0, 1, 0}));
        std::vector<uint8_t> truncated(bytes.begin(), bytes.end() - 2);
        expect_throw<std::invalid_argument>([&] { b2co::RoaringBitmap<uint32_t> bad(truncated.data(), truncated.size(), stream); });
    }

    // ---- HyperLogLog<int64_t>: estimate within 3 standard errors ----
    {
        auto h = b2co::HyperLogLog<int64_t>::CreateWithSketchSizeKB(64, stream);
        CHECK(h.SketchSizeKB() == 64);
        std::vector<int64_t> keys(1000000);
        for (auto& k : keys) k = int64_t(gen() % 300000);
        std::unordered_set<int64_t> distinct(keys.begin(), keys.end());
        DeviceBuffer<int64_t> dk(keys);
        h.Add(dk.p, b2co::Extent<size_t>{keys.size()}, stream);
        double est = double(h.Estimate(stream)), truth = double(distinct.size());
        CHECK(std::abs(est - truth) <= 3 * 1.04 / 256.0 * truth);
        expect_throw<std::invalid_argument>([&] { b2co::HyperLogLog<int64_t>::CreateWithPrecision(12); });
    }

    std::printf("cpp api test ok\n");
    return 0;
}
