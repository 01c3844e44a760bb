// bloom.cu -- BloomFilter<Key> with any BloomFilterPolicy of 32-bit words
// (bloom_filter_policy.h:42-181): blocks of W uint32 words, xxh64 of the key,
// block = mulhi32(upper hash, numBlocks), PatternBits / W bits per word, bit b
// of word w at (salt[w * bitsPerWord + b] * lower hash) >> 27.
//
// B200 design for the default policy (W = 8, one bit per word): a block is
// exactly one 32-byte L2 sector.  Add stages the block's 8 word bits in shared
// memory and ORs the whole sector into the filter with one TMA bulk reduction
// (cp.reduce.async.bulk .or.b32); the alternative issues them as four 64-bit
// atomic ORs that need no return value (RED), all to that one sector, with
// lanes of a warp that hit the same block merged first (match_any).  Contains reads the sector with two
// 16-byte loads.  Other policies run one key per thread: W/2 64-bit REDs (one
// 32-bit RED for W = 1) and vector loads of the block.  Merge/Intersect stream
// 16 bytes per lane (4 when the word count is not a multiple of 4).
#include <new>

#include "b2co_host.h"

using namespace b2co;

namespace {

// The policy's 64-entry salt table (bloom_filter_policy.h:170-178).  The first
// eight are the split-block Bloom filter salts of the Parquet specification,
// all the default policy uses; a policy with bitsPerWord bits per word takes
// salt[w * bitsPerWord + b] for bit b of word w.
__constant__ uint32_t kSalts[64] = {
    0x47b6137bu, 0x44974d91u, 0x8824ad5bu, 0xa2b7289du, 0x705495c7u, 0x2df1424bu, 0x9efc4947u, 0x5c6bfb31u,
    0xb24bcdffu, 0xb6843d6du, 0x6db04543u, 0x3a12efddu, 0xb0ddd463u, 0x8d22f6e7u, 0xb82f1e53u, 0x7db9f86bu,
    0xc7afe639u, 0xfb135cd7u, 0x693256e1u, 0x9466d871u, 0x23d3d02fu, 0x6461d049u, 0x66a91621u, 0xbaa3006fu,
    0x52fb8d99u, 0x3ea88b4fu, 0x0f470cfdu, 0xb1db79a5u, 0x9809fcd1u, 0xbced4445u, 0x2eb7c737u, 0x2cea6803u,
    0x156f1955u, 0x8813c027u, 0xa26819f9u, 0x4c3b57bdu, 0x7df94487u, 0xb975e769u, 0xb8f20cb5u, 0x5c9e2e77u,
    0x5fb1735fu, 0x3a6f759bu, 0x3c090923u, 0xfced424du, 0xa187a6a9u, 0x6f070a41u, 0x2c85233bu, 0x7e62258bu,
    0x2771ef17u, 0x13bbf093u, 0x4ff059e5u, 0xe3ce3d0fu, 0xf1b4789fu, 0x9fbb6173u, 0x6a320cf5u, 0x1be2c481u,
    0x7ba8222bu, 0x6fd619b3u, 0x7b1bbf0du, 0x8b8993adu, 0x448eca95u, 0x82ab09d9u, 0x2ce53909u, 0x4f548685u};

template <int KB>
__device__ __forceinline__ void locate(uint64_t key, uint64_t seed, uint32_t nblocks, uint32_t& block, uint32_t& lower)
{
    uint64_t h = xxh64<KB>(key, seed);
    block = uint32_t((uint64_t(uint32_t(h >> 32)) * nblocks) >> 32);
    lower = uint32_t(h);
}

__device__ __forceinline__ uint32_t word_bit(int w, uint32_t lower) { return 1u << ((kSalts[w] * lower) >> 27); }

template <int KB>
__device__ __forceinline__ uint64_t load_key(void const* keys, uint64_t i)
{
    if constexpr (KB == 8) return __ldg(reinterpret_cast<unsigned long long const*>(keys) + i);
    else return __ldg(reinterpret_cast<uint32_t const*>(keys) + i);
}

template <int KB>
__global__ void __launch_bounds__(256) k_bloom_add(uint32_t* words, uint32_t nblocks, uint64_t seed, void const* keys,
                                                   uint8_t const* stencil, uint64_t n)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t base = uint64_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        uint64_t i = base + (threadIdx.x & 31);
        bool live = i < n && (!stencil || stencil[i]);
        uint32_t block = 0xffffffffu, lower = 0;
        if (live) locate<KB>(load_key<KB>(keys, i), seed, nblocks, block, lower);
        uint32_t pat[8];
#pragma unroll
        for (int w = 0; w < 8; ++w) pat[w] = live ? word_bit(w, lower) : 0u;
        // lanes sharing a block OR their patterns together; the lowest lane issues the REDs
        uint32_t peers = __match_any_sync(0xffffffffu, block);
        uint32_t const lane = threadIdx.x & 31;
        if (__popc(peers) > 1) {
#pragma unroll
            for (int w = 0; w < 8; ++w) {
                uint32_t acc = pat[w];
                for (uint32_t m = peers; m; m &= m - 1) acc |= __shfl_sync(peers, pat[w], __ffs(m) - 1);
                pat[w] = acc;
            }
        }
        if (live && lane == uint32_t(__ffs(peers) - 1)) {
            unsigned long long* p = reinterpret_cast<unsigned long long*>(words + uint64_t(block) * 8);
#pragma unroll
            for (int q = 0; q < 4; ++q) atomicOr(p + q, (unsigned long long)pat[2 * q] | ((unsigned long long)pat[2 * q + 1] << 32));
        }
    }
}

// Bulk-reduction Add (default policy): every key writes its block's eight
// words (one bit each) to its own 32-byte slot in shared memory and the TMA
// unit ORs the whole 32-byte block into the filter with one
// cp.reduce.async.bulk .or.b32 (element-wise atomic in L2), instead of four
// 64-bit atomics from the SM.  Each thread double-buffers its slot: before
// reusing a slot it waits until the bulk operation that read it has read it.
// Slots per thread: bulk reductions a thread may have in flight.
#ifndef B2CO_BLOOM_BULK_DEPTH
#define B2CO_BLOOM_BULK_DEPTH 2
#endif

template <int KB>
__global__ void __launch_bounds__(256) k_bloom_add_bulk(uint32_t* words, uint32_t nblocks, uint64_t seed,
                                                        void const* keys, uint8_t const* stencil, uint64_t n)
{
    constexpr int D = B2CO_BLOOM_BULK_DEPTH;
    static_assert(D >= 2 && D <= 8, "bulk depth");
    __shared__ alignas(128) uint32_t stage[D][256][8];
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    uint32_t b = 0;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (stencil && !stencil[i]) continue;
        uint32_t block, lower;
        locate<KB>(load_key<KB>(keys, i), seed, nblocks, block, lower);
        // the bulk operation issued D keys ago read this slot: wait for that read
        asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(D - 1) : "memory");
        uint32_t* slot = stage[b][threadIdx.x];
#pragma unroll
        for (int q = 0; q < 2; ++q)
            reinterpret_cast<uint4*>(slot)[q] = make_uint4(word_bit(4 * q, lower), word_bit(4 * q + 1, lower),
                                                           word_bit(4 * q + 2, lower), word_bit(4 * q + 3, lower));
        fence_proxy_async();  // the generic-proxy writes above precede the bulk read
        asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.or.b32 [%0], [%1], 32;" ::"l"(
                         words + uint64_t(block) * 8),
                     "r"(smem_u32(slot))
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        b = b + 1 == D ? 0 : b + 1;
    }
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // every reduction done before the slots go away
}

template <int KB>
__global__ void __launch_bounds__(256) k_bloom_contains(uint32_t const* words, uint32_t nblocks, uint64_t seed,
                                                        void const* keys, uint8_t const* stencil, uint8_t* out,
                                                        uint64_t n)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint8_t r = 0;
        if (!stencil || stencil[i]) {
            uint32_t block, lower;
            locate<KB>(load_key<KB>(keys, i), seed, nblocks, block, lower);
            uint4 const* p = reinterpret_cast<uint4 const*>(words + uint64_t(block) * 8);
            uint4 a = __ldg(p), b = __ldg(p + 1);
            uint32_t const w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            bool all = true;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                uint32_t bit = word_bit(j, lower);
                all &= (w[j] & bit) == bit;
            }
            r = all;
        }
        out[i] = r;
    }
}

// ---- any other policy: W words per block, bpw bits per word ------------------

__device__ __forceinline__ uint32_t policy_pattern(uint32_t w, uint32_t bpw, uint32_t lower)
{
    uint32_t pat = 0;
    for (uint32_t b = 0; b < bpw; ++b) pat |= 1u << ((kSalts[w * bpw + b] * lower) >> 27);
    return pat;
}

template <int KB, int W>
__global__ void __launch_bounds__(256) k_bloom_add_policy(uint32_t* words, uint32_t nblocks, uint32_t bpw,
                                                          uint64_t seed, void const* keys, uint8_t const* stencil,
                                                          uint64_t n)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (stencil && !stencil[i]) continue;
        uint32_t block, lower;
        locate<KB>(load_key<KB>(keys, i), seed, nblocks, block, lower);
        uint32_t* blk = words + uint64_t(block) * W;
        if constexpr (W == 1) {
            atomicOr(blk, policy_pattern(0, bpw, lower));
        } else {  // a block of W >= 2 words starts on an 8-byte boundary: 64-bit REDs
#pragma unroll
            for (int q = 0; q < W / 2; ++q)
                atomicOr(reinterpret_cast<unsigned long long*>(blk) + q,
                         (unsigned long long)policy_pattern(2 * q, bpw, lower) |
                             ((unsigned long long)policy_pattern(2 * q + 1, bpw, lower) << 32));
        }
    }
}

template <int W>
__device__ __forceinline__ void load_block(uint32_t const* blk, uint32_t (&w)[W])
{
    if constexpr (W % 4 == 0) {
#pragma unroll
        for (int q = 0; q < W / 4; ++q) {
            uint4 v = __ldg(reinterpret_cast<uint4 const*>(blk) + q);
            w[4 * q] = v.x, w[4 * q + 1] = v.y, w[4 * q + 2] = v.z, w[4 * q + 3] = v.w;
        }
    } else if constexpr (W == 2) {
        uint2 v = __ldg(reinterpret_cast<uint2 const*>(blk));
        w[0] = v.x, w[1] = v.y;
    } else {
        w[0] = __ldg(blk);
    }
}

template <int KB, int W>
__global__ void __launch_bounds__(256) k_bloom_contains_policy(uint32_t const* words, uint32_t nblocks, uint32_t bpw,
                                                               uint64_t seed, void const* keys, uint8_t const* stencil,
                                                               uint8_t* out, uint64_t n)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint8_t r = 0;
        if (!stencil || stencil[i]) {
            uint32_t block, lower;
            locate<KB>(load_key<KB>(keys, i), seed, nblocks, block, lower);
            uint32_t w[W];
            load_block<W>(words + uint64_t(block) * W, w);
            bool all = true;
#pragma unroll
            for (int j = 0; j < W; ++j) {
                uint32_t const pat = policy_pattern(j, bpw, lower);
                all &= (w[j] & pat) == pat;
            }
            r = all;
        }
        out[i] = r;
    }
}

template <int OP>  // 0 = or, 1 = and; filters whose word count is not a multiple of 4
__global__ void __launch_bounds__(256) k_bloom_combine32(uint32_t* dst, uint32_t const* src, uint64_t n)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = OP == 0 ? (dst[i] | __ldg(src + i)) : (dst[i] & __ldg(src + i));
}

template <int OP>  // 0 = or, 1 = and
__global__ void __launch_bounds__(256) k_bloom_combine(uint4* dst, uint4 const* src, uint64_t n16)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n16; i += stride) {
        uint4 a = dst[i], b = __ldg(src + i);
        if (OP == 0) a = make_uint4(a.x | b.x, a.y | b.y, a.z | b.z, a.w | b.w);
        else a = make_uint4(a.x & b.x, a.y & b.y, a.z & b.z, a.w & b.w);
        dst[i] = a;
    }
}

cudaStream_t cs(b2co_stream s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

struct b2co_bloom {
    uint32_t* words = nullptr;
    int add_mode = B2CO_BLOOM_ADD_BULK;  // default-policy Add: bulk reductions (measured faster) or 64-bit atomics
    uint64_t num_blocks = 0;
    uint32_t key_bytes = 0;
    uint64_t seed = 0;
    uint32_t wpb = 8;           // WordsPerBlock
    uint32_t pattern_bits = 8;  // PatternBits
    uint64_t num_words() const { return num_blocks * wpb; }
    bool default_policy() const { return wpb == 8 && pattern_bits == 8; }
};

namespace {

int check(b2co_bloom const* f)
{
    if (!f || !f->words) return fail(B2CO_ELOGIC, "BloomFilter: a moved-from filter cannot participate");
    return B2CO_OK;
}

// ValidateCompatible (bloom_filter_query.inl:197-215).
int check_pair(b2co_bloom const* a, b2co_bloom const* b, char const* op)
{
    if (int st = check(a)) return st;
    if (int st = check(b)) return st;
    if (a->num_blocks != b->num_blocks)
        return fail(B2CO_EINVAL, std::string("BloomFilter::") + op + ": filters have different block extents");
    if (a->seed != b->seed || a->key_bytes != b->key_bytes || a->wpb != b->wpb || a->pattern_bits != b->pattern_bits)
        return fail(B2CO_EINVAL, std::string("BloomFilter::") + op + ": filters have different policies");
    return B2CO_OK;
}

template <int KB>
int launch_add_policy(b2co_bloom* f, void const* keys, uint8_t const* stencil, uint64_t n, cudaStream_t s)
{
    void (*k)(uint32_t*, uint32_t, uint32_t, uint64_t, void const*, uint8_t const*, uint64_t) = nullptr;
    switch (f->wpb) {
        case 1: k = k_bloom_add_policy<KB, 1>; break;
        case 2: k = k_bloom_add_policy<KB, 2>; break;
        case 4: k = k_bloom_add_policy<KB, 4>; break;
        case 8: k = k_bloom_add_policy<KB, 8>; break;
        case 16: k = k_bloom_add_policy<KB, 16>; break;
        default: k = k_bloom_add_policy<KB, 32>; break;
    }
    k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(f->words, uint32_t(f->num_blocks),
                                                           f->pattern_bits / f->wpb, f->seed, keys, stencil, n);
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

template <int KB>
int launch_contains_policy(b2co_bloom* f, void const* keys, uint8_t const* stencil, uint8_t* out, uint64_t n,
                           cudaStream_t s)
{
    void (*k)(uint32_t const*, uint32_t, uint32_t, uint64_t, void const*, uint8_t const*, uint8_t*, uint64_t) =
        nullptr;
    switch (f->wpb) {
        case 1: k = k_bloom_contains_policy<KB, 1>; break;
        case 2: k = k_bloom_contains_policy<KB, 2>; break;
        case 4: k = k_bloom_contains_policy<KB, 4>; break;
        case 8: k = k_bloom_contains_policy<KB, 8>; break;
        case 16: k = k_bloom_contains_policy<KB, 16>; break;
        default: k = k_bloom_contains_policy<KB, 32>; break;
    }
    k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(f->words, uint32_t(f->num_blocks),
                                                           f->pattern_bits / f->wpb, f->seed, keys, stencil, out, n);
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

int add_impl(b2co_bloom* f, void const* keys, uint8_t const* stencil, bool use_stencil, uint64_t n, cudaStream_t s)
{
    if (int st = check(f)) return st;
    if (n == 0) return B2CO_OK;
    if (!keys) return fail(B2CO_EINVAL, "BloomFilter::Add: keys must not be null when keyNum is non-zero");
    if (use_stencil && !stencil)
        return fail(B2CO_EINVAL, "BloomFilter::AddIf: stencil must not be null when keyNum is non-zero");
    if (!f->default_policy())
        return f->key_bytes == 8 ? launch_add_policy<8>(f, keys, stencil, n, s) : launch_add_policy<4>(f, keys, stencil, n, s);
    void (*k)(uint32_t*, uint32_t, uint64_t, void const*, uint8_t const*, uint64_t) = nullptr;
    if (f->add_mode == B2CO_BLOOM_ADD_BULK) k = f->key_bytes == 8 ? k_bloom_add_bulk<8> : k_bloom_add_bulk<4>;
    else k = f->key_bytes == 8 ? k_bloom_add<8> : k_bloom_add<4>;
    k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(f->words, uint32_t(f->num_blocks), f->seed, keys, stencil,
                                                           n);
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

int contains_impl(b2co_bloom* f, void const* keys, uint8_t const* stencil, bool use_stencil, uint8_t* out, uint64_t n,
                  cudaStream_t s)
{
    if (int st = check(f)) return st;
    if (n == 0) return B2CO_OK;
    if (!keys) return fail(B2CO_EINVAL, "BloomFilter::Contains: keys must not be null when keyNum is non-zero");
    if (!out) return fail(B2CO_EINVAL, "BloomFilter::Contains: outputValues must not be null when keyNum is non-zero");
    if (use_stencil && !stencil)
        return fail(B2CO_EINVAL, "BloomFilter::ContainsIf: stencil must not be null when keyNum is non-zero");
    if (!f->default_policy())
        return f->key_bytes == 8 ? launch_contains_policy<8>(f, keys, stencil, out, n, s)
                                 : launch_contains_policy<4>(f, keys, stencil, out, n, s);
    void (*k)(uint32_t const*, uint32_t, uint64_t, void const*, uint8_t const*, uint8_t*, uint64_t) =
        f->key_bytes == 8 ? k_bloom_contains<8> : k_bloom_contains<4>;
    k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(f->words, uint32_t(f->num_blocks), f->seed, keys, stencil,
                                                           out, n);
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

template <int OP>
int combine(b2co_bloom* f, b2co_bloom const* o, cudaStream_t s, char const* name)
{
    if (int st = check_pair(f, o, name)) return st;
    if (f == o) return B2CO_OK;
    uint64_t const nw = f->num_words();
    if (nw % 4 == 0) {
        uint64_t const n16 = nw / 4;
        auto k = k_bloom_combine<OP>;
        k<<<grid_for((void const*)k, 256, n16, 256), 256, 0, s>>>(reinterpret_cast<uint4*>(f->words),
                                                                  reinterpret_cast<uint4 const*>(o->words), n16);
    } else {
        auto k = k_bloom_combine32<OP>;
        k<<<grid_for((void const*)k, 256, nw, 256), 256, 0, s>>>(f->words, o->words, nw);
    }
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

int sync(cudaStream_t s)
{
    B2CO_CUDA(cudaStreamSynchronize(s));
    return B2CO_OK;
}

}  // namespace

extern "C" {

int b2co_bloom_create(uint64_t num_blocks, uint32_t key_bytes, uint64_t seed, b2co_stream stream, b2co_bloom** out)
{
    return b2co_bloom_create_policy(num_blocks, key_bytes, seed, 8, 8, stream, out);
}

int b2co_bloom_create_policy(uint64_t num_blocks, uint32_t key_bytes, uint64_t seed, uint32_t words_per_block,
                             uint32_t pattern_bits, b2co_stream stream, b2co_bloom** out)
{
    if (!out) return fail(B2CO_EINVAL, "null output");
    *out = nullptr;
    if (num_blocks == 0) return fail(B2CO_EINVAL, "BloomFilter: numBlocks must be greater than zero");
    if (num_blocks > 0xffffffffull)
        return fail(B2CO_ERANGE, "BloomFilter: numBlocks exceeds the supported block-index range");
    if (key_bytes != 4 && key_bytes != 8) return fail(B2CO_EINVAL, "BloomFilter: key_bytes must be 4 or 8");
    // the policy constructor's static_asserts (bloom_filter_policy.h:60-86) for 32-bit words
    uint32_t const w = words_per_block, p = pattern_bits;
    if (w == 0 || (w & (w - 1)) != 0 || w > 32)
        return fail(B2CO_EINVAL, "BloomFilter: WordsPerBlock must be a power of two not above 32");
    if (p < w || p > 64 || p > 32 * w || p % w != 0)
        return fail(B2CO_EINVAL, "BloomFilter: PatternBits must be a multiple of WordsPerBlock in [WordsPerBlock, "
                                 "min(64, 32 * WordsPerBlock)]");
    auto* f = new (std::nothrow) b2co_bloom;
    if (!f) return fail(B2CO_ENOMEM, "host allocation failed");
    f->num_blocks = num_blocks;
    f->key_bytes = key_bytes;
    f->seed = seed;
    f->wpb = w;
    f->pattern_bits = p;
    cudaError_t e = cudaMalloc(&f->words, f->num_words() * 4);
    if (e != cudaSuccess) {
        delete f;
        return cuda_fail(e, "BloomFilter allocation");
    }
    if (int st = b2co_bloom_clear(f, stream)) {
        b2co_bloom_destroy(f);
        return st;
    }
    *out = f;
    return B2CO_OK;
}

int b2co_bloom_destroy(b2co_bloom* f)
{
    if (!f) return B2CO_OK;
    if (f->words) cudaFree(f->words);
    delete f;
    return B2CO_OK;
}

int b2co_bloom_data(b2co_bloom const* f, uint32_t** words)
{
    if (int st = check(f)) return st;
    if (!words) return fail(B2CO_EINVAL, "null output");
    *words = f->words;
    return B2CO_OK;
}

int b2co_bloom_num_blocks(b2co_bloom const* f, uint64_t* nb)
{
    if (int st = check(f)) return st;
    if (!nb) return fail(B2CO_EINVAL, "null output");
    *nb = f->num_blocks;
    return B2CO_OK;
}

int b2co_bloom_policy(b2co_bloom const* f, uint32_t* words_per_block, uint32_t* pattern_bits)
{
    if (int st = check(f)) return st;
    if (!words_per_block || !pattern_bits) return fail(B2CO_EINVAL, "null output");
    *words_per_block = f->wpb;
    *pattern_bits = f->pattern_bits;
    return B2CO_OK;
}

int b2co_bloom_clear_async(b2co_bloom* f, b2co_stream s)
{
    if (int st = check(f)) return st;
    B2CO_CUDA(cudaMemsetAsync(f->words, 0, f->num_words() * 4, cs(s)));
    return B2CO_OK;
}

int b2co_bloom_clear(b2co_bloom* f, b2co_stream s)
{
    if (int st = b2co_bloom_clear_async(f, s)) return st;
    return sync(cs(s));
}

int b2co_bloom_add_async(b2co_bloom* f, void const* keys, uint64_t n, b2co_stream s)
{
    return add_impl(f, keys, nullptr, false, n, cs(s));
}

int b2co_bloom_add(b2co_bloom* f, void const* keys, uint64_t n, b2co_stream s)
{
    if (int st = add_impl(f, keys, nullptr, false, n, cs(s))) return st;
    return sync(cs(s));
}

int b2co_bloom_add_if_async(b2co_bloom* f, void const* keys, uint8_t const* stencil, uint64_t n, b2co_stream s)
{
    return add_impl(f, keys, stencil, true, n, cs(s));
}

int b2co_bloom_add_if(b2co_bloom* f, void const* keys, uint8_t const* stencil, uint64_t n, b2co_stream s)
{
    if (int st = add_impl(f, keys, stencil, true, n, cs(s))) return st;
    return sync(cs(s));
}

int b2co_bloom_contains_async(b2co_bloom* f, void const* keys, uint8_t* out, uint64_t n, b2co_stream s)
{
    return contains_impl(f, keys, nullptr, false, out, n, cs(s));
}

int b2co_bloom_contains(b2co_bloom* f, void const* keys, uint8_t* out, uint64_t n, b2co_stream s)
{
    if (int st = contains_impl(f, keys, nullptr, false, out, n, cs(s))) return st;
    return sync(cs(s));
}

int b2co_bloom_contains_if_async(b2co_bloom* f, void const* keys, uint8_t const* stencil, uint8_t* out, uint64_t n,
                                 b2co_stream s)
{
    return contains_impl(f, keys, stencil, true, out, n, cs(s));
}

int b2co_bloom_contains_if(b2co_bloom* f, void const* keys, uint8_t const* stencil, uint8_t* out, uint64_t n,
                           b2co_stream s)
{
    if (int st = contains_impl(f, keys, stencil, true, out, n, cs(s))) return st;
    return sync(cs(s));
}

int b2co_bloom_merge_async(b2co_bloom* f, b2co_bloom const* o, b2co_stream s) { return combine<0>(f, o, cs(s), "Merge"); }

int b2co_bloom_merge(b2co_bloom* f, b2co_bloom const* o, b2co_stream s)
{
    if (int st = combine<0>(f, o, cs(s), "Merge")) return st;
    return sync(cs(s));
}

int b2co_bloom_intersect_async(b2co_bloom* f, b2co_bloom const* o, b2co_stream s)
{
    return combine<1>(f, o, cs(s), "Intersect");
}

int b2co_bloom_intersect(b2co_bloom* f, b2co_bloom const* o, b2co_stream s)
{
    if (int st = combine<1>(f, o, cs(s), "Intersect")) return st;
    return sync(cs(s));
}

}  // extern "C"

extern "C" {

int b2co_bloom_set_add_mode(b2co_bloom* f, int mode)
{
    if (int st = check(f)) return st;
    if (mode != B2CO_BLOOM_ADD_ATOMIC && mode != B2CO_BLOOM_ADD_BULK) return fail(B2CO_EINVAL, "unknown Add mode");
    f->add_mode = mode;
    return B2CO_OK;
}

}  // extern "C"
