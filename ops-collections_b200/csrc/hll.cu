// hll.cu -- HyperLogLog<Key> for int32/int64 keys, precision 13..18
// (include/hyperloglog.h, hyperloglog_ref.h:30-47, detail/hyperloglog/*).
//
// Register rule: h = xxh64(key, seed 0); index = top p bits; rank =
// clz((h << p) | 2^(p-1)) + 1 (so rank <= 65 - p); register = max(register,
// rank).  Registers are bytes, register i at byte i (four per 32-bit word).
//
// B200 design: Add keeps a private copy of the registers in shared memory
// (p <= 17: 8..128 KiB per CTA of 1024 threads), reads each key once from HBM
// in 16-byte loads, and raises a shared register with a compare-and-swap loop
// only when the new rank is larger (after warm-up almost never).  Each CTA then folds its copy into the
// global registers with a per-byte max (__vmaxu4) CAS on words that changed.
// p = 18 (256 KiB) exceeds shared memory and updates the global registers
// directly, with the same read-before-CAS filter.  Estimate builds the 65-bin
// rank histogram on the device and finishes with the HLL++ finalizer on the host.
#include <cmath>
#include <cstring>
#include <limits>
#include <new>

#include "b2co_host.h"
#include "hllpp_data.inc"

using namespace b2co;

namespace {

constexpr int kBins = 65;

template <int KB>
__device__ __forceinline__ uint64_t load_key(void const* keys, uint64_t i)
{
    if constexpr (KB == 8) return __ldg(reinterpret_cast<unsigned long long const*>(keys) + i);
    else return __ldg(reinterpret_cast<uint32_t const*>(keys) + i);
}

template <int KB>
__device__ __forceinline__ void hll_locate(uint64_t key, uint32_t p, uint32_t& index, uint32_t& rank)
{
    uint64_t h = xxh64<KB>(key, 0);
    index = uint32_t(h >> (64 - p));
    uint64_t tail = (h << p) | (1ull << (p - 1));
    rank = uint32_t(__clzll((long long)tail)) + 1u;
}

// Raise byte `index` of the register words to at least `rank`.
__device__ __forceinline__ void raise_register(uint32_t* words, uint32_t index, uint32_t rank)
{
    uint32_t* w = words + (index >> 2);
    uint32_t const shift = (index & 3u) * 8u;
    uint32_t observed = *reinterpret_cast<volatile uint32_t*>(w);
    while (((observed >> shift) & 255u) < rank) {
        uint32_t desired = (observed & ~(255u << shift)) | (rank << shift);
        uint32_t prev = atomicCAS(w, observed, desired);
        if (prev == observed) break;
        observed = prev;
    }
}

// Fold a register word into the global registers with a per-byte maximum.
__device__ __forceinline__ void fold_word(uint32_t* g, uint32_t mine)
{
    uint32_t observed = *reinterpret_cast<volatile uint32_t*>(g);
    for (;;) {
        uint32_t desired = __vmaxu4(observed, mine);
        if (desired == observed) return;
        uint32_t prev = atomicCAS(g, observed, desired);
        if (prev == observed) return;
        observed = prev;
    }
}

// Precision as a compile-time constant: the index and rank shifts become
// immediates.
template <int KB, int P>
__device__ __forceinline__ void hll_locate_p(uint64_t key, uint32_t& index, uint32_t& rank)
{
    uint64_t const h = xxh64<KB>(key, 0);
    index = uint32_t(h >> (64 - P));
    rank = uint32_t(__clzll((long long)((h << P) | (1ull << (P - 1))))) + 1u;
}

constexpr int kHllBlock = 1024;

// Add for p <= 17 with 16-byte key loads: a CTA of 1024 threads keeps one
// private register copy (2^P bytes of shared memory), so at p = 16 two CTAs
// fill an SM's 64 warps.  Keys before the first 16-byte boundary (`head`) and
// after the last whole vector go one per thread.
template <int KB, int P>
__global__ void __launch_bounds__(kHllBlock, P <= 16 ? 2 : 1)
    k_hll_add_vec(uint32_t* regs, void const* keys, uint64_t n, uint64_t head)
{
    extern __shared__ uint32_t sk[];
    constexpr uint32_t kWords = (1u << P) / 4;
    constexpr int V = 16 / KB;        // keys per 16-byte load
    constexpr int U = KB == 8 ? 2 : 1;  // loads in flight per thread
    for (uint32_t i = threadIdx.x; i < kWords; i += kHllBlock) sk[i] = 0;
    __syncthreads();
    uint64_t const tid = uint64_t(blockIdx.x) * kHllBlock + threadIdx.x;
    uint64_t const stride = uint64_t(gridDim.x) * kHllBlock;
    auto add = [&](uint64_t key) {
        uint32_t x, r;
        hll_locate_p<KB, P>(key, x, r);
        raise_register(sk, x, r);  // a word load decides; a byte load measured 3.5x slower
    };
    uint64_t const body = head < n ? n - head : 0;
    uint64_t const nvec = body / V;
    uint64_t const tail0 = head + nvec * V;
    for (uint64_t i = tid; i < head && i < n; i += stride) add(load_key<KB>(keys, i));
    for (uint64_t i = tail0 + tid; i < n; i += stride) add(load_key<KB>(keys, i));
    uint4 const* vk = reinterpret_cast<uint4 const*>(static_cast<char const*>(keys) + head * KB);
    auto add_vec = [&](uint4 q) {
        if constexpr (KB == 8) {
            add(uint64_t(q.x) | (uint64_t(q.y) << 32));
            add(uint64_t(q.z) | (uint64_t(q.w) << 32));
        } else {
            add(q.x);
            add(q.y);
            add(q.z);
            add(q.w);
        }
    };
    uint64_t v = tid;
    for (; v + (U - 1) * stride < nvec; v += U * stride) {
        uint4 q[U];
#pragma unroll
        for (int j = 0; j < U; ++j) q[j] = __ldcs(vk + v + j * stride);
#pragma unroll
        for (int j = 0; j < U; ++j) add_vec(q[j]);
    }
    for (; v < nvec; v += stride) add_vec(__ldcs(vk + v));
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < kWords; w += kHllBlock) {
        uint32_t const mine = sk[w];
        if (mine) fold_word(regs + w, mine);
    }
}

template <int KB>
__global__ void __launch_bounds__(256) k_hll_add_global(uint32_t* regs, uint32_t p, void const* keys, uint64_t n)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t x, r;
        hll_locate<KB>(load_key<KB>(keys, i), p, x, r);
        raise_register(regs, x, r);
    }
}

__global__ void __launch_bounds__(256) k_hll_merge(uint32_t* dst, uint32_t const* src, uint32_t words)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x)
        dst[i] = __vmaxu4(dst[i], src[i]);
}

__global__ void __launch_bounds__(256) k_hll_histogram(uint32_t const* regs, uint32_t words, unsigned int* hist)
{
    __shared__ unsigned int h[kBins];
    for (int b = threadIdx.x; b < kBins; b += blockDim.x) h[b] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) {
        uint32_t w = regs[i];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            uint32_t r = (w >> (8 * b)) & 255u;
            atomicAdd(&h[r < kBins ? r : kBins - 1], 1u);
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kBins; b += blockDim.x)
        if (h[b]) atomicAdd(hist + b, h[b]);
}

cudaStream_t cs(b2co_stream s) { return reinterpret_cast<cudaStream_t>(s); }

double const (*points_for(uint32_t p, uint32_t& n))[2]
{
    switch (p) {
        case 13: n = sizeof(kHllppP13) / sizeof(kHllppP13[0]); return kHllppP13;
        case 14: n = sizeof(kHllppP14) / sizeof(kHllppP14[0]); return kHllppP14;
        case 15: n = sizeof(kHllppP15) / sizeof(kHllppP15[0]); return kHllppP15;
        case 16: n = sizeof(kHllppP16) / sizeof(kHllppP16[0]); return kHllppP16;
        case 17: n = sizeof(kHllppP17) / sizeof(kHllppP17[0]); return kHllppP17;
        case 18: n = sizeof(kHllppP18) / sizeof(kHllppP18[0]); return kHllppP18;
    }
    n = 0;
    return nullptr;
}

// Separate contiguous views of the raw estimates and biases (built once).
struct BiasViews {
    double raw[6][256];
    double bias[6][256];
    uint32_t n[6];
    BiasViews()
    {
        for (uint32_t p = 13; p <= 18; ++p) {
            uint32_t cnt;
            auto pts = points_for(p, cnt);
            n[p - 13] = cnt;
            for (uint32_t i = 0; i < cnt && i < 256; ++i) {
                raw[p - 13][i] = pts[i][0];
                bias[p - 13][i] = pts[i][1];
            }
        }
    }
};
BiasViews const& views()
{
    static BiasViews v;
    return v;
}

// HLL++ finalizer (detail/hyperloglog/finalizer.h:46-151): linear counting
// below 2.5 m, the empirical threshold, 6-nearest-neighbour bias
// interpolation below 5 m, the raw estimate otherwise.
uint64_t finalize(uint32_t p, double z, int v)
{
    if (z == 0.0) return std::numeric_limits<uint64_t>::max();
    int const m = 1 << p;
    double alpha;
    switch (m) {
        case 16: alpha = 0.673; break;
        case 32: alpha = 0.697; break;
        case 64: alpha = 0.709; break;
        default: alpha = 0.7213 / (1.0 + 1.079 / m);
    }
    double e = alpha * m * m / z;
    bool correct = false;
    if (v > 0) {
        double const h = m * std::log(double(m) / v);
        if (e <= 2.5 * m) return uint64_t(std::round(h));
        if (p < 19) {
            if (h <= kHllppThreshold[p - 13]) e = h;
            else correct = true;
        }
    } else if (p < 19) {
        correct = true;
    }
    if (correct && e < 5.0 * m) {
        auto const& V = views();
        double const* raw = V.raw[p - 13];
        double const* bias = V.bias[p - 13];
        int const np = int(V.n[p - 13]);
        int left = 0, right = np - 1, anchor = -1;
        while (left <= right) {
            int mid = left + (right - left) / 2;
            if (raw[mid] < e) left = mid + 1;
            else if (raw[mid] > e) right = mid - 1;
            else {
                anchor = mid;
                break;
            }
        }
        if (anchor < 0) anchor = left;
        constexpr int k = 6;
        int low = std::max(std::min(anchor - k + 1, np - k), 0);
        int high = std::min(low + k, np);
        auto dist = [&](int i) { double d = e - raw[i]; return d * d; };
        while (high < np && dist(high) < dist(low)) ++low, ++high;
        double sum = 0.0;
        for (int i = low; i < high; ++i) sum += bias[i];
        e -= sum / (high - low);
    }
    if (e >= double(std::numeric_limits<uint64_t>::max())) return std::numeric_limits<uint64_t>::max();
    return uint64_t(std::round(e));
}

}  // namespace

struct b2co_hll {
    uint32_t* regs = nullptr;       // 2^p bytes
    unsigned int* d_hist = nullptr; // 65 bins
    unsigned int* h_hist = nullptr; // pinned mirror
    uint32_t precision = 0;
    uint32_t key_bytes = 0;
    int device = -1;
};

namespace {

// Validate (hyperloglog.inl:204-213): storage present and the owner device current.
int check(b2co_hll const* h)
{
    if (!h || !h->regs) return fail(B2CO_ELOGIC, "HyperLogLog: moved-from or uninitialized sketch");
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != h->device) return fail(B2CO_EINVAL, "HyperLogLog: current device differs from owner device");
    return B2CO_OK;
}

int add_launch(b2co_hll* h, void const* keys, uint64_t n, cudaStream_t s)
{
    uint32_t const p = h->precision;
    if (p <= 17) {
        using AddFn = void (*)(uint32_t*, void const*, uint64_t, uint64_t);
        static AddFn const fns[2][5] = {
            {k_hll_add_vec<4, 13>, k_hll_add_vec<4, 14>, k_hll_add_vec<4, 15>, k_hll_add_vec<4, 16>,
             k_hll_add_vec<4, 17>},
            {k_hll_add_vec<8, 13>, k_hll_add_vec<8, 14>, k_hll_add_vec<8, 15>, k_hll_add_vec<8, 16>,
             k_hll_add_vec<8, 17>}};
        // the shared-memory opt-in is a per-device function attribute: set it on
        // every launch (it costs about a microsecond), cache only the occupancy
        constexpr int kDevices = 64;
        static int per_sm_cache[kDevices][2][5] = {};
        int const ki = h->key_bytes == 8, pi = int(p) - 13, dev = h->device;
        AddFn const k = fns[ki][pi];
        size_t const smem = size_t(1) << p;
        B2CO_CUDA(cudaFuncSetAttribute((void const*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        int per_sm = dev >= 0 && dev < kDevices ? per_sm_cache[dev][ki][pi] : 0;
        if (!per_sm) {
            B2CO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (void const*)k, kHllBlock, smem));
            if (per_sm < 1) per_sm = 1;
            if (dev >= 0 && dev < kDevices) per_sm_cache[dev][ki][pi] = per_sm;
        }
        uint64_t const want = (n + uint64_t(kHllBlock) * 16 - 1) / (uint64_t(kHllBlock) * 16);  // >= ~16 keys a thread
        uint64_t const cap = uint64_t(per_sm) * sm_count();
        uint32_t const grid = uint32_t(want < 1 ? 1 : (want < cap ? want : cap));
        // keys up to the first 16-byte boundary go one per thread
        uintptr_t const addr = reinterpret_cast<uintptr_t>(keys);
        uint64_t const head = ((16 - addr % 16) % 16) / h->key_bytes;
        k<<<grid, kHllBlock, smem, s>>>(h->regs, keys, n, head);
    } else {
        void (*k)(uint32_t*, uint32_t, void const*, uint64_t) =
            h->key_bytes == 8 ? k_hll_add_global<8> : k_hll_add_global<4>;
        k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(h->regs, p, keys, n);
    }
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

}  // namespace

extern "C" {

// CreateWithSketchSizeKB (hyperloglog.inl:115-123).
int b2co_hll_precision_for_sketch_kb(uint32_t kb, uint32_t* precision)
{
    if (!precision) return fail(B2CO_EINVAL, "null output");
    if (kb < 8 || kb > 256 || (kb & (kb - 1)) != 0) return fail(B2CO_EINVAL, "HyperLogLog: invalid sketch size");
    uint32_t p = 13;
    while ((1u << p) < kb * 1024u) ++p;
    *precision = p;
    return B2CO_OK;
}

// CreateWithStandardDeviation (hyperloglog.inl:132-141).
int b2co_hll_precision_for_deviation(double d, uint32_t* precision)
{
    if (!precision) return fail(B2CO_EINVAL, "null output");
    if (!std::isfinite(d) || d <= 0) return fail(B2CO_EINVAL, "HyperLogLog: invalid deviation");
    for (uint32_t p = 13; p <= 18; ++p)
        if (1.04 / std::sqrt(double(1u << p)) <= d) {
            *precision = p;
            return B2CO_OK;
        }
    return fail(B2CO_EINVAL, "HyperLogLog: deviation requires more than 256 KiB");
}

int b2co_hll_create(uint32_t precision, uint32_t key_bytes, b2co_stream stream, b2co_hll** out)
{
    if (!out) return fail(B2CO_EINVAL, "null output");
    *out = nullptr;
    if (precision < 13 || precision > 18) return fail(B2CO_EINVAL, "HyperLogLog: precision must be in [13, 18]");
    if (key_bytes != 4 && key_bytes != 8) return fail(B2CO_EINVAL, "HyperLogLog supports int32_t and int64_t");
    auto* h = new (std::nothrow) b2co_hll;
    if (!h) return fail(B2CO_ENOMEM, "host allocation failed");
    h->precision = precision;
    h->key_bytes = key_bytes;
    cudaGetDevice(&h->device);
    cudaError_t e = cudaMalloc(&h->regs, size_t(1) << precision);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_hist, kBins * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_hist, kBins * sizeof(unsigned int));
    if (e != cudaSuccess) {
        b2co_hll_destroy(h);
        return cuda_fail(e, "HyperLogLog allocation");
    }
    if (int st = b2co_hll_clear(h, stream)) {
        b2co_hll_destroy(h);
        return st;
    }
    *out = h;
    return B2CO_OK;
}

int b2co_hll_destroy(b2co_hll* h)
{
    if (!h) return B2CO_OK;
    if (h->regs) cudaFree(h->regs);
    if (h->d_hist) cudaFree(h->d_hist);
    if (h->h_hist) cudaFreeHost(h->h_hist);
    delete h;
    return B2CO_OK;
}

int b2co_hll_data(b2co_hll const* h, uint8_t const** regs)
{
    if (!h || !h->regs) return fail(B2CO_ELOGIC, "HyperLogLog: moved-from or uninitialized sketch");
    if (!regs) return fail(B2CO_EINVAL, "null output");
    *regs = reinterpret_cast<uint8_t const*>(h->regs);
    return B2CO_OK;
}

int b2co_hll_precision(b2co_hll const* h, uint32_t* p)
{
    if (!h || !h->regs) return fail(B2CO_ELOGIC, "HyperLogLog: moved-from or uninitialized sketch");
    if (!p) return fail(B2CO_EINVAL, "null output");
    *p = h->precision;
    return B2CO_OK;
}

int b2co_hll_clear(b2co_hll* h, b2co_stream s)
{
    if (int st = check(h)) return st;
    B2CO_CUDA(cudaMemsetAsync(h->regs, 0, size_t(1) << h->precision, cs(s)));
    B2CO_CUDA(cudaStreamSynchronize(cs(s)));
    return B2CO_OK;
}

int b2co_hll_add_async(b2co_hll* h, void const* keys, uint64_t n, b2co_stream s)
{
    if (int st = check(h)) return st;
    if (n == 0) return B2CO_OK;
    if (!keys || reinterpret_cast<uintptr_t>(keys) % h->key_bytes != 0)
        return fail(B2CO_EINVAL, "HyperLogLog: invalid input pointer or size");
    return add_launch(h, keys, n, cs(s));
}

int b2co_hll_add(b2co_hll* h, void const* keys, uint64_t n, b2co_stream s)
{
    if (int st = b2co_hll_add_async(h, keys, n, s)) return st;
    B2CO_CUDA(cudaStreamSynchronize(cs(s)));
    return B2CO_OK;
}

// Merge = bytewise max (hyperloglog.inl:315-326; incompatible -> EINVAL).
int b2co_hll_merge(b2co_hll* h, b2co_hll const* o, b2co_stream s)
{
    if (int st = check(h)) return st;
    if (int st = check(o)) return st;
    if (h->precision != o->precision || h->device != o->device)
        return fail(B2CO_EINVAL, "HyperLogLog: incompatible sketches");
    if (h != o) {
        uint32_t words = (1u << h->precision) / 4;
        k_hll_merge<<<grid_for((void const*)k_hll_merge, 256, words, 256), 256, 0, cs(s)>>>(h->regs, o->regs, words);
        B2CO_CUDA(cudaGetLastError());
    }
    B2CO_CUDA(cudaStreamSynchronize(cs(s)));
    return B2CO_OK;
}

int b2co_hll_histogram(b2co_hll const* h, b2co_stream s, uint32_t* host_hist)
{
    if (int st = check(h)) return st;
    if (!host_hist) return fail(B2CO_EINVAL, "null output");
    cudaStream_t c = cs(s);
    uint32_t words = (1u << h->precision) / 4;
    B2CO_CUDA(cudaMemsetAsync(h->d_hist, 0, kBins * sizeof(unsigned int), c));
    k_hll_histogram<<<grid_for((void const*)k_hll_histogram, 256, words, 256 * 16), 256, 0, c>>>(h->regs, words,
                                                                                               h->d_hist);
    B2CO_CUDA(cudaGetLastError());
    B2CO_CUDA(cudaMemcpyAsync(h->h_hist, h->d_hist, kBins * sizeof(unsigned int), cudaMemcpyDeviceToHost, c));
    B2CO_CUDA(cudaStreamSynchronize(c));
    std::memcpy(host_hist, h->h_hist, kBins * sizeof(uint32_t));
    return B2CO_OK;
}

int b2co_hll_finalize(uint32_t p, uint32_t const* hist, uint64_t* estimate)
{
    if (!hist || !estimate) return fail(B2CO_EINVAL, "null argument");
    if (p < 13 || p > 18) return fail(B2CO_EINVAL, "HyperLogLog: precision must be in [13, 18]");
    double z = 0.0;
    for (int r = 0; r < kBins; ++r) z += std::ldexp(double(hist[r]), -r);
    *estimate = finalize(p, z, int(hist[0]));
    return B2CO_OK;
}

// Estimate (hyperloglog.inl:328-345).
int b2co_hll_estimate(b2co_hll const* h, b2co_stream s, uint64_t* estimate)
{
    if (!estimate) return fail(B2CO_EINVAL, "null output");
    uint32_t hist[kBins];
    if (int st = b2co_hll_histogram(h, s, hist)) return st;
    return b2co_hll_finalize(h->precision, hist, estimate);
}

int b2co_hll_bias_data(uint32_t p, double const** raw, double const** bias, uint32_t* points, double* threshold)
{
    if (p < 13 || p > 18) return fail(B2CO_EINVAL, "HyperLogLog: precision must be in [13, 18]");
    auto const& V = views();
    if (raw) *raw = V.raw[p - 13];
    if (bias) *bias = V.bias[p - 13];
    if (points) *points = V.n[p - 13];
    if (threshold) *threshold = kHllppThreshold[p - 13];
    return B2CO_OK;
}

}  // extern "C"
