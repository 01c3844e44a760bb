// runtime.cu -- error state, launch geometry and the capacity prime rule.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "b2co_host.h"

namespace b2co {

static thread_local std::string g_last_error;

int fail(int status, std::string const& msg)
{
    g_last_error = msg;
    return status;
}

int cuda_fail(cudaError_t e, char const* what)
{
    return fail(e == cudaErrorMemoryAllocation ? B2CO_ENOMEM : B2CO_ECUDA,
                std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

namespace {
bool capturing(cudaStream_t s)
{
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return st != cudaStreamCaptureStatusNone;
}
}  // namespace

int ScratchOrder::begin(cudaStream_t s)
{
    if (capturing(s)) return B2CO_OK;
    if (!done) B2CO_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    if (used) B2CO_CUDA(cudaStreamWaitEvent(s, done, 0));
    return B2CO_OK;
}

int ScratchOrder::end(cudaStream_t s)
{
    if (capturing(s) || !done) return B2CO_OK;
    B2CO_CUDA(cudaEventRecord(done, s));
    used = true;
    return B2CO_OK;
}

void ScratchOrder::release()
{
    if (done) cudaEventDestroy(done);
    done = nullptr;
    used = false;
}

int sm_count()
{
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

uint32_t grid_for(void const* kernel, uint32_t block, uint64_t work, uint64_t per_block)
{
    // resident blocks per SM of this kernel at this block size, cached
    struct Occ {
        void const* kernel;
        uint32_t block;
        int per_sm;
    };
    static std::mutex mu;
    static std::vector<Occ> occ;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> g(mu);
        for (auto& e : occ)
            if (e.kernel == kernel && e.block == block) per_sm = e.per_sm;
        if (per_sm == 0) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, int(block), 0) != cudaSuccess ||
                per_sm <= 0)
                per_sm = 1;
            occ.push_back(Occ{kernel, block, per_sm});
        }
    }
    uint64_t want = per_block ? (work + per_block - 1) / per_block : 1;
    uint64_t cap = uint64_t(per_sm) * uint64_t(sm_count());
    if (want < 1) want = 1;
    return uint32_t(want < cap ? want : cap);
}

static std::atomic<unsigned long long> g_wait_ns{1000000000ull};
static std::atomic<unsigned int> g_wait_probe{0};

WaitCtl wait_ctl(unsigned int* status) { return WaitCtl{status, g_wait_ns.load(), g_wait_probe.load()}; }

// ---------------------------------------------------------------------------
// Capacity primes.  The reference's table (include/utility/prime.h:15, 140,741
// entries) follows a rule: 2, 3, 5, 7, 11, 13; then the smallest prime >=
// previous + 6, with 151 listed right after 149, up to 131,101; from there the
// smallest prime >= previous + 2^17.  The library regenerates the table from
// that rule instead of shipping it; tests pin the result against the
// reference's table by hash.
// ---------------------------------------------------------------------------

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return uint64_t((unsigned __int128)a * b % m); }

static bool is_prime(uint64_t n)
{
    static uint64_t const bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return false;
    for (uint64_t p : bases) {
        if (n == p) return true;
        if (n % p == 0) return false;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) d >>= 1, ++s;
    for (uint64_t a : bases) {
        uint64_t x = 1, base = a % n, e = d;
        while (e) {
            if (e & 1) x = mulmod(x, base, n);
            base = mulmod(base, base, n);
            e >>= 1;
        }
        if (x == 1 || x == n - 1) continue;
        bool composite = true;
        for (int r = 1; r < s && composite; ++r) {
            x = mulmod(x, x, n);
            if (x == n - 1) composite = false;
        }
        if (composite) return false;
    }
    return true;
}

static uint64_t next_prime(uint64_t n)
{
    while (!is_prime(n)) ++n;
    return n;
}

static constexpr size_t kPrimeCount = 140741;

static std::vector<uint64_t> const& primes()
{
    static std::vector<uint64_t> table;
    static std::once_flag once;
    std::call_once(once, [] {
        table.reserve(kPrimeCount);
        for (uint64_t p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull}) table.push_back(p);
        uint64_t p = 13;
        while (p <= 131072) {
            p = next_prime(p + 6);
            table.push_back(p);
            if (p == 149) table.push_back(p = 151);
        }
        while (table.size() < kPrimeCount) table.push_back(p = next_prime(p + 131072));
    });
    return table;
}

uint64_t prime_at_least(uint64_t n)
{
    auto const& t = primes();
    auto it = std::lower_bound(t.begin(), t.end(), n);
    return it == t.end() ? 0 : *it;
}

uint64_t prime_table_last() { return primes().back(); }

}  // namespace b2co

extern "C" {

const char* b2co_last_error(void) { return b2co::g_last_error.c_str(); }

const char* b2co_status_string(int s)
{
    switch (s) {
        case B2CO_OK: return "ok";
        case B2CO_EINVAL: return "invalid argument";
        case B2CO_ERANGE: return "length error";
        case B2CO_ENOMEM: return "out of memory";
        case B2CO_ECUDA: return "CUDA runtime error";
        case B2CO_ETIMEOUT: return "device wait timed out";
        case B2CO_ELOGIC: return "logic error";
        case B2CO_EOVERFLOW: return "overflow error";
    }
    return "unknown status";
}

const char* b2co_version(void) { return "b2co 0.1 (sm_100a)"; }

int b2co_set_l2_fetch_granularity(uint32_t bytes, uint64_t* applied)
{
    if (bytes != 0 && bytes != 32 && bytes != 64 && bytes != 128)
        return b2co::fail(B2CO_EINVAL, "L2 fetch granularity must be 32, 64 or 128 bytes");
    if (bytes) B2CO_CUDA(cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, bytes));
    if (applied) {
        size_t v = 0;
        B2CO_CUDA(cudaDeviceGetLimit(&v, cudaLimitMaxL2FetchGranularity));
        *applied = v;
    }
    return B2CO_OK;
}

int b2co_debug_set_wait(uint64_t limit_ns, int probe_timeout)
{
    b2co::g_wait_ns.store(limit_ns ? limit_ns : 1000000000ull);
    b2co::g_wait_probe.store(probe_timeout ? 1u : 0u);
    return B2CO_OK;
}

// Host evaluation of the device-side key primitives (include/b2co/device.cuh).
int b2co_probe_hash(uint32_t hash, uint32_t key_bytes, uint64_t key_bits, uint32_t seed, uint32_t* out)
{
    if (!out) return b2co::fail(B2CO_EINVAL, "output is null");
    if (hash > B2CO_HASH_XXH64) return b2co::fail(B2CO_EINVAL, "unknown hash");
    if (hash == B2CO_HASH_FMIX && key_bytes == 2) return b2co::fail(B2CO_EINVAL, "the Fmix hashes take 4 or 8 bytes");
    switch (key_bytes) {
        case 2: *out = b2co::probe_hash<2>(hash, key_bits & 0xffffu, seed); break;
        case 4: *out = b2co::probe_hash<4>(hash, key_bits & 0xffffffffu, seed); break;
        case 8: *out = b2co::probe_hash<8>(hash, key_bits, seed); break;
        default: return b2co::fail(B2CO_EINVAL, "key_bytes must be 2, 4 or 8");
    }
    return B2CO_OK;
}

int b2co_key_equal(uint32_t key_kind, uint32_t key_bytes, uint64_t a_bits, uint64_t b_bits, int* equal)
{
    if (!equal) return b2co::fail(B2CO_EINVAL, "output is null");
    if (key_kind > B2CO_KEY_FLOAT) return b2co::fail(B2CO_EINVAL, "unknown key kind");
    uint64_t const m = key_bytes >= 8 ? ~0ull : ((1ull << (8 * key_bytes)) - 1ull);
    a_bits &= m;
    b_bits &= m;
    bool r = false;
    switch (key_bytes) {
        case 2: r = key_kind ? b2co::key_equal<2, true>(a_bits, b_bits) : b2co::key_equal<2, false>(a_bits, b_bits); break;
        case 4: r = key_kind ? b2co::key_equal<4, true>(a_bits, b_bits) : b2co::key_equal<4, false>(a_bits, b_bits); break;
        case 8: r = key_kind ? b2co::key_equal<8, true>(a_bits, b_bits) : b2co::key_equal<8, false>(a_bits, b_bits); break;
        default: return b2co::fail(B2CO_EINVAL, "key_bytes must be 2, 4 or 8");
    }
    *equal = r ? 1 : 0;
    return B2CO_OK;
}

// MakeValidExtent (include/detail/extent/extent.inl:20-62).
int b2co_oa_valid_capacity(uint64_t requested, uint32_t b, uint32_t probing, uint64_t* capacity)
{
    if (!capacity) return b2co::fail(B2CO_EINVAL, "capacity output is null");
    if (b != 1 && b != 2 && b != 4 && b != 5 && b != 8) return b2co::fail(B2CO_EINVAL, "unsupported bucket size");
    uint64_t m = requested > 1 ? requested : 1;
    uint64_t size = m / b + (m % b != 0);
    if (probing == B2CO_PROBE_DOUBLE) {
        uint64_t p = b2co::prime_at_least(size);
        if (p == 0) return b2co::fail(B2CO_EINVAL, "Invalid input Extent");
        *capacity = p * b;
    } else if (probing == B2CO_PROBE_LINEAR) {
        *capacity = (size + (requested == 0)) * b;
    } else {
        return b2co::fail(B2CO_EINVAL, "unknown probing scheme");
    }
    return B2CO_OK;
}

}  // extern "C"
