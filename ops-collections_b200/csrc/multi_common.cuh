// multi_common.cuh -- building blocks of the multi-containers (StaticMultiset,
// StaticMultimap): an order-preserving device-wide scan, a key -> count table,
// and a stable LSD radix-sort pass.
//
// * Tile scan: items are processed in tiles of kTile; a first pass reduces each
//   tile (k_tile_reduce), one block scans the tile sums (k_scan_tiles), and a
//   second pass recomputes the items and hands each its exclusive prefix in
//   input order (k_tile_apply).  Items are read striped (coalesced) and ranked
//   round by round, so ranks follow the input order exactly.
// * Key table: a power-of-two open-addressing table of distinct keys with a
//   32-bit count per key, linear probing from fmix(key); the empty key marks a
//   free slot; keys are claimed with a 32/64-bit CAS.  It is never more than
//   half full, so every probe ends at the key or at a free slot.
// * Radix pass: a stable counting-sort pass over one byte of a 16-byte record,
//   histogram per tile -> exclusive scan (digit-major) -> in-order scatter with
//   per-warp match_any ranking.
#pragma once

#include "b2co_host.h"

namespace b2co {
namespace multi {

constexpr int kThreads = 256;
constexpr int kRounds = 8;                    // items per thread per tile
constexpr uint64_t kTile = kThreads * kRounds;  // 2048

// Block-wide exclusive scan of one value per thread; *total gets the block sum.
__device__ __forceinline__ uint64_t block_excl_scan(uint64_t v, uint64_t* total)
{
    __shared__ uint64_t warp_sums[kThreads / 32];
    __shared__ uint64_t block_total;
    uint32_t const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= uint32_t(d)) incl += o;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint64_t s = lane < kThreads / 32 ? warp_sums[lane] : 0;
        uint64_t si = s;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint64_t o = __shfl_up_sync(0xffffffffu, si, d);
            if (lane >= uint32_t(d)) si += o;
        }
        if (lane < kThreads / 32) warp_sums[lane] = si - s;
        if (lane == kThreads / 32 - 1) block_total = si;
    }
    __syncthreads();
    uint64_t const r = warp_sums[warp] + incl - v;
    *total = block_total;
    __syncthreads();  // the shared words are reused by the next call
    return r;
}

// Pass 1: per-tile sums of f(i) for i < n.
template <class F>
__global__ void __launch_bounds__(kThreads) k_tile_reduce(F f, uint64_t n, uint64_t* tile_sums)
{
    uint64_t const base = uint64_t(blockIdx.x) * kTile;
    uint64_t s = 0;
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        uint64_t const i = base + uint64_t(r) * kThreads + threadIdx.x;
        if (i < n) s += f(i);
    }
    uint64_t total;
    block_excl_scan(s, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Pass 2 (one block): exclusive scan of the tile sums in place; *total = sum.
__global__ void __launch_bounds__(kThreads) k_scan_tiles(uint64_t* sums, uint64_t ntiles, uint64_t* total)
{
    uint64_t carry = 0;
    for (uint64_t base = 0; base < ntiles; base += kThreads) {
        uint64_t const i = base + threadIdx.x;
        uint64_t const v = i < ntiles ? sums[i] : 0;
        uint64_t chunk;
        uint64_t const e = block_excl_scan(v, &chunk);
        if (i < ntiles) sums[i] = carry + e;
        carry += chunk;
    }
    if (threadIdx.x == 0) *total = carry;
}

// Pass 3: every item gets its exclusive prefix in input order: act(i, value, prefix).
template <class F, class A>
__global__ void __launch_bounds__(kThreads) k_tile_apply(F f, A act, uint64_t n, uint64_t const* tile_offsets)
{
    uint64_t const base = uint64_t(blockIdx.x) * kTile;
    uint64_t carry = tile_offsets[blockIdx.x];
#pragma unroll 1
    for (int r = 0; r < kRounds; ++r) {
        uint64_t const i = base + uint64_t(r) * kThreads + threadIdx.x;
        uint64_t const v = i < n ? f(i) : 0;
        uint64_t round_total;
        uint64_t const e = block_excl_scan(v, &round_total);
        if (i < n) act(i, v, carry + e);
        carry += round_total;
    }
}

// Host driver of the three passes.  `scratch` holds ceil(n / kTile) + 1 words;
// returns the total through *total_dev (device) -- the caller reads it when needed.
template <class F, class A>
int tile_scan(F f, A act, uint64_t n, uint64_t* scratch, bool apply, cudaStream_t s)
{
    uint64_t const tiles = (n + kTile - 1) / kTile;
    uint64_t* total = scratch + tiles;
    if (n == 0) {
        B2CO_CUDA(cudaMemsetAsync(total, 0, sizeof(uint64_t), s));
        return B2CO_OK;
    }
    k_tile_reduce<<<uint32_t(tiles), kThreads, 0, s>>>(f, n, scratch);
    k_scan_tiles<<<1, kThreads, 0, s>>>(scratch, tiles, total);
    if (apply) k_tile_apply<<<uint32_t(tiles), kThreads, 0, s>>>(f, act, n, scratch);
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

inline uint64_t scan_scratch_words(uint64_t n) { return (n + kTile - 1) / kTile + 1; }

struct NoAct {
    __device__ void operator()(uint64_t, uint64_t, uint64_t) const {}
};

// ---- key -> count table --------------------------------------------------------

template <int KB>
using KeyWord = typename std::conditional<KB == 4, unsigned int, unsigned long long>::type;

template <int KB>
struct KeyTable {
    KeyWord<KB>* keys;
    uint32_t* counts;
    uint32_t* offsets;  // multimap: first CSR position of the key's values
    uint64_t mask;      // table size - 1 (a power of two)
    KeyWord<KB> empty;
};

template <int KB>
__device__ __forceinline__ uint64_t table_hash(KeyWord<KB> k)
{
    if constexpr (KB == 4) return fmix32(k, 0);
    else return fmix64(k, 0);
}

// Adds `delta` to the key's count, claiming a slot if the key is new; its slot.
template <int KB>
__device__ __forceinline__ uint64_t table_add(KeyTable<KB> const& t, KeyWord<KB> k, uint32_t delta)
{
    uint64_t s = table_hash<KB>(k) & t.mask;
    for (;;) {
        KeyWord<KB> cur = t.keys[s];
        if (cur == t.empty) cur = atomicCAS(t.keys + s, t.empty, k);
        if (cur == t.empty || cur == k) {
            atomicAdd(t.counts + s, delta);
            return s;
        }
        s = (s + 1) & t.mask;
    }
}

// The key's slot, or ~0 when absent (the table is at most half full).
template <int KB>
__device__ __forceinline__ uint64_t table_find(KeyTable<KB> const& t, KeyWord<KB> k)
{
    if (k == t.empty) return ~0ull;
    uint64_t s = table_hash<KB>(k) & t.mask;
    for (;;) {
        KeyWord<KB> const cur = t.keys[s];
        if (cur == k) return s;
        if (cur == t.empty) return ~0ull;
        s = (s + 1) & t.mask;
    }
}

template <int KB>
__global__ void __launch_bounds__(256) k_table_clear(KeyTable<KB> t)
{
    uint64_t const n = t.mask + 1, stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        t.keys[i] = t.empty;
        t.counts[i] = 0;
    }
}

inline uint64_t table_size_for(uint64_t max_keys)
{
    uint64_t t = 64;
    while (t < 2 * max_keys) t <<= 1;
    return t;
}

// ---- stable LSD radix pass over a byte of a 16-byte record --------------------

struct alignas(16) Record {
    unsigned long long vbits;  // order-preserving value bits
    uint32_t slot;             // key table slot
    uint32_t pad;
};

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr uint64_t kSortTile = uint64_t(kSortThreads) * kSortRounds;  // 4096

__device__ __forceinline__ uint32_t record_digit(Record const& r, int pass, int value_bytes)
{
    return pass < value_bytes ? uint32_t(r.vbits >> (8 * pass)) & 0xffu : (r.slot >> (8 * (pass - value_bytes))) & 0xffu;
}

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(Record const* in, uint64_t n, int pass, int value_bytes,
                                                             uint64_t ntiles, uint64_t* hist)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    uint64_t const base = uint64_t(blockIdx.x) * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
        uint64_t const i = base + uint64_t(r) * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(h + record_digit(in[i], pass, value_bytes), 1u);
    }
    __syncthreads();
    hist[uint64_t(threadIdx.x) * ntiles + blockIdx.x] = h[threadIdx.x];  // digit-major
}

__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(Record const* in, Record* out, uint64_t n, int pass,
                                                                int value_bytes, uint64_t ntiles,
                                                                uint64_t const* offsets)
{
    constexpr int kWarps = kSortThreads / 32;
    __shared__ uint64_t running[256];
    __shared__ uint32_t wcnt[kWarps][256];
    uint32_t const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    running[threadIdx.x] = offsets[uint64_t(threadIdx.x) * ntiles + blockIdx.x];
    uint64_t const base = uint64_t(blockIdx.x) * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        uint64_t const i = base + uint64_t(r) * kSortThreads + threadIdx.x;
        bool const live = i < n;
        Record rec{};
        uint32_t d = 256;  // no digit
        if (live) {
            rec = in[i];
            d = record_digit(rec, pass, value_bytes);
        }
        uint32_t const peers = __match_any_sync(0xffffffffu, d);
        uint32_t const below = peers & ((1u << lane) - 1u);
        if (live && below == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (live) {
            uint64_t pos = running[d] + __popc(below);
            for (uint32_t w = 0; w < warp; ++w) pos += wcnt[w][d];
            out[pos] = rec;
        }
        __syncthreads();
        uint32_t add = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) add += wcnt[w][threadIdx.x];
        running[threadIdx.x] += add;
        __syncthreads();
    }
}

}  // namespace multi
}  // namespace b2co
