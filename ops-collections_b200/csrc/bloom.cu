// bloom.cu -- BloomFilter<Key> with any BloomFilterPolicy of 32-bit words
// (bloom_filter_policy.h:42-181): blocks of W uint32 words, xxh64 of the key,
// block = mulhi32(upper hash, numBlocks), PatternBits / W bits per word, bit b
// of word w at (salt[w * bitsPerWord + b] * lower hash) >> 27.
//
// B200 design for the default policy (W = 8, one bit per word): a block is
// exactly one 32-byte L2 sector.  Three Adds set the same bits:
//  * bulk: the block's 8 word bits are staged in shared memory and the whole
//    sector is ORed into the filter with one TMA bulk reduction
//    (cp.reduce.async.bulk .or.b32);
//  * atomic: four 64-bit atomic ORs without a return value (RED) to that one
//    sector, lanes of a warp that hit the same block merged first (match_any);
//  * routed (large batches on large filters): keys are sorted by 128 KiB filter
//    slice through a workspace, each slice is built in shared memory and ORed
//    in with bulk reductions (see the partitioned Add below).
// Contains reads the sector with two 16-byte loads, four keys per thread.
// Other policies run one key per thread: W/2 64-bit REDs (one 32-bit RED for
// W = 1) and vector loads of the block.  Merge/Intersect stream 16 bytes per
// lane (4 when the word count is not a multiple of 4).
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

// ---- partitioned Add (default policy, large batches) ------------------------
// The route-then-apply plan of bloom_filter_launch.inl:131-240 with B200
// shapes.  The filter is cut into slices of kSliceBlocks blocks (128 KiB); a
// key's record is its block within the slice (high 32 bits) and the lower
// hash half (low 32 bits).  Each of R route CTAs owns one contiguous chunk of
// the batch.
//   count   : CTA c counts its chunk's records per slice -> counts[c][s];
//   colscan : per slice, the exclusive prefix over the CTAs (in place) and the
//             slice's total;
//   scan    : slice offsets into the record workspace (records of a slice are
//             contiguous, CTA by CTA);
//   route   : CTA c hashes its chunk a tile at a time, sorts the tile's
//             records by slice in shared memory and writes each slice's run at
//             its own running cursor -- no global atomics, and writes leave in
//             runs rather than one record at a time;
//   apply   : one CTA per slice ORs the slice's records into a shared-memory
//             copy of the slice and reduces the whole copy into the filter with
//             TMA bulk ORs (element-wise atomic in L2, so concurrent Adds on
//             other streams stay correct).
// DRAM traffic per key is the key twice and a record written and read back
// (8 + 8 + 8 + 8 bytes), against two scattered 32-byte block transfers per key
// otherwise.
constexpr uint32_t kSliceBlocks = 4096;
constexpr uint32_t kMaxSlices = 2048;  // filters up to 256 MiB take this path
constexpr int kRouteThreads = 1024;
constexpr int kRouteKeys = 8;  // keys per thread and tile
constexpr int kRouteTile = kRouteThreads * kRouteKeys;
constexpr int kApplyThreads = 1024;

// Chunk of route CTA c: whole tiles, the last chunk possibly short.
__device__ __forceinline__ void route_chunk(uint64_t n, uint32_t c, uint32_t nctas, uint64_t& begin, uint64_t& end)
{
    uint64_t const tiles = (n + kRouteTile - 1) / kRouteTile;
    uint64_t const per = (tiles + nctas - 1) / nctas;
    begin = uint64_t(c) * per * kRouteTile;
    end = begin + per * kRouteTile;
    if (begin > n) begin = n;
    if (end > n) end = n;
}

template <int KB>
__global__ void __launch_bounds__(1024, 2) k_bloom_count(uint32_t nblocks, uint64_t seed, void const* keys,
                                                     uint8_t const* stencil, uint64_t n, uint32_t nslices,
                                                     uint32_t nctas, uint32_t* counts)
{
    __shared__ uint32_t hist[kMaxSlices];
    for (uint32_t i = threadIdx.x; i < nslices; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    uint64_t begin, end;
    route_chunk(n, blockIdx.x, nctas, begin, end);
    constexpr int kKeys = 8;  // keys loaded before any is hashed
    for (uint64_t i0 = begin + threadIdx.x; i0 < end; i0 += uint64_t(kKeys) * blockDim.x) {
        uint64_t key[kKeys];
        bool live[kKeys];
#pragma unroll
        for (int j = 0; j < kKeys; ++j) {
            uint64_t const i = i0 + uint64_t(j) * blockDim.x;
            live[j] = i < end && (!stencil || stencil[i]);
            key[j] = live[j] ? load_key<KB>(keys, i) : 0;
        }
#pragma unroll
        for (int j = 0; j < kKeys; ++j) {
            uint32_t block, lower;
            locate<KB>(key[j], seed, nblocks, block, lower);
            if (live[j]) atomicAdd(&hist[block / kSliceBlocks], 1u);
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nslices; i += blockDim.x) counts[uint64_t(blockIdx.x) * nslices + i] = hist[i];
}

// Per slice (one thread each): exclusive prefix of its counts over the route
// CTAs, in place, and the slice's total.
__global__ void __launch_bounds__(256) k_bloom_colscan(uint32_t* counts, uint32_t nslices, uint32_t nctas,
                                                       uint32_t* totals)
{
    uint32_t const sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= nslices) return;
    uint32_t run = 0;
    for (uint32_t c = 0; c < nctas; ++c) {
        uint32_t* p = counts + uint64_t(c) * nslices + sl;
        uint32_t const v = *p;
        *p = run;
        run += v;
    }
    totals[sl] = run;
}

// Exclusive scan of the slice totals (one CTA): offsets[0..nslices].
__global__ void __launch_bounds__(1024) k_bloom_scan(uint32_t const* totals, uint32_t nslices, uint32_t* offsets)
{
    __shared__ uint32_t warp_tot[32];
    constexpr int kPer = kMaxSlices / 1024;
    uint32_t const t = threadIdx.x, lane = t & 31, warp = t >> 5;
    uint32_t v[kPer], sum = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        uint32_t const i = t * kPer + j;
        v[j] = i < nslices ? totals[i] : 0u;
        sum += v[j];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t const o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= uint32_t(d)) incl += o;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t const w = warp_tot[lane];
        uint32_t wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t const o = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= uint32_t(d)) wi += o;
        }
        warp_tot[lane] = wi - w;  // exclusive prefix of the warp totals
    }
    __syncthreads();
    uint32_t run = warp_tot[warp] + incl - sum;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        uint32_t const i = t * kPer + j;
        if (i <= nslices) offsets[i] = run;
        run += v[j];
    }
    if (t == 1023 && nslices == kMaxSlices) offsets[nslices] = run;
}

// Shared memory of one route CTA: the next tile's keys (8 bytes a key), the
// tile's records and their destinations, then per slice the tile's count, its
// offset in the tile, its run's global start, the CTA's running cursor and the
// slice's end in the workspace.
__host__ __device__ constexpr uint32_t route_bins(uint32_t nslices) { return (nslices + 31) & ~31u; }
__host__ __device__ constexpr size_t route_smem(uint32_t nslices)
{
    return size_t(kRouteTile) * (8 + 8 + 4) + size_t(route_bins(nslices)) * 4 * 5 + (kRouteThreads / 32 + 1) * 4;
}

template <int KB>
__device__ __forceinline__ void cp_async_key(void* dst, void const* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(KB) : "memory");
}

template <int KB>
__global__ void __launch_bounds__(kRouteThreads) k_bloom_route(uint32_t nblocks, uint64_t seed, void const* keys,
                                                               uint8_t const* stencil, uint64_t n, uint32_t nslices,
                                                               uint32_t nctas, uint32_t const* prefix,
                                                               uint32_t const* offsets, unsigned long long* recs)
{
    extern __shared__ __align__(16) unsigned char route_smem_[];
    auto* kbuf = reinterpret_cast<unsigned long long*>(route_smem_);  // one 8-byte cell a key
    auto* stage = kbuf + kRouteTile;
    auto* stage_at = reinterpret_cast<uint32_t*>(stage + kRouteTile);
    uint32_t const nbins = route_bins(nslices);
    uint32_t* hist = stage_at + kRouteTile;
    uint32_t* loff = hist + nbins;
    uint32_t* gbase = loff + nbins;
    uint32_t* gcur = gbase + nbins;
    uint32_t* gend = gcur + nbins;
    uint32_t* warp_tot = gend + nbins;  // kRouteThreads / 32 warp sums, then the tile's total
    uint32_t const t = threadIdx.x, lane = t & 31, warp = t >> 5;
    constexpr uint32_t kNone = 0xffffffffu;
    constexpr int kWarps = kRouteThreads / 32;
    constexpr int kPer = kMaxSlices / kRouteThreads;
    for (uint32_t i = t; i < nslices; i += kRouteThreads) {
        gcur[i] = offsets[i] + prefix[uint64_t(blockIdx.x) * nslices + i];
        gend[i] = offsets[i + 1];
    }
    uint64_t begin, end;
    route_chunk(n, blockIdx.x, nctas, begin, end);
    // a thread copies its own keys of the next tile into its own cells while the
    // CTA works on this tile (cp.async), so key loads never stall a tile
    auto prefetch = [&](uint64_t b) {
#pragma unroll
        for (int j = 0; j < kRouteKeys; ++j) {
            uint64_t const i = b + uint64_t(j) * kRouteThreads + t;
            if (i < end) cp_async_key<KB>(kbuf + j * kRouteThreads + t, static_cast<char const*>(keys) + i * KB);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (begin < end) prefetch(begin);
    for (uint64_t base = begin; base < end; base += kRouteTile) {
        for (uint32_t i = t; i < nslices; i += kRouteThreads) hist[i] = 0;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        unsigned long long rec[kRouteKeys];
        uint32_t where[kRouteKeys];  // slice << 16 | rank in the tile, or kNone
        uint64_t key[kRouteKeys];
        bool live[kRouteKeys];
#pragma unroll
        for (int j = 0; j < kRouteKeys; ++j) {
            uint64_t const i = base + uint64_t(j) * kRouteThreads + t;
            live[j] = i < end && (!stencil || stencil[i]);
            unsigned long long const cell = kbuf[j * kRouteThreads + t];
            key[j] = live[j] ? (KB == 8 ? cell : uint64_t(uint32_t(cell))) : 0;
        }
        if (base + kRouteTile < end) prefetch(base + kRouteTile);  // each thread reuses only its own cells
        __syncthreads();
        // a record's rank within its slice comes from the shared histogram
#pragma unroll
        for (int j = 0; j < kRouteKeys; ++j) {
            uint32_t block, lower;
            locate<KB>(key[j], seed, nblocks, block, lower);
            rec[j] = (uint64_t(block % kSliceBlocks) << 32) | lower;
            where[j] = block / kSliceBlocks;
        }
#pragma unroll
        for (int j = 0; j < kRouteKeys; ++j)
            where[j] = live[j] ? (where[j] << 16) | atomicAdd(&hist[where[j]], 1u) : kNone;
        __syncthreads();
        // the tile's offsets per slice (exclusive scan, kPer slices per thread);
        // each slice's run starts at the CTA's cursor for it
        uint32_t v[kPer], sum = 0;
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            uint32_t const i = t * kPer + q;
            v[q] = i < nslices ? hist[i] : 0u;
            sum += v[q];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t const o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= uint32_t(d)) incl += o;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t const w = lane < kWarps ? warp_tot[lane] : 0u;
            uint32_t wi = w;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                uint32_t const o = __shfl_up_sync(0xffffffffu, wi, d);
                if (lane >= uint32_t(d)) wi += o;
            }
            if (lane < kWarps) warp_tot[lane] = wi - w;
            if (lane == 31) warp_tot[kWarps] = wi;  // the tile's record count
        }
        __syncthreads();
        uint32_t run = warp_tot[warp] + incl - sum;
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            uint32_t const i = t * kPer + q;
            if (i < nslices) {
                loff[i] = run;
                gbase[i] = gcur[i];
                gcur[i] += v[q];
            }
            run += v[q];
        }
        __syncthreads();
        // records sorted by slice in shared memory, each with its destination; a
        // record never passes its slice's end (only keys changed between the
        // count and this pass could ask it to)
#pragma unroll
        for (int j = 0; j < kRouteKeys; ++j) {
            if (where[j] == kNone) continue;
            uint32_t const sl = where[j] >> 16, r = where[j] & 0xffffu, g = gbase[sl] + r;
            stage[loff[sl] + r] = rec[j];
            stage_at[loff[sl] + r] = g < gend[sl] ? g : kNone;
        }
        __syncthreads();
        // each slice's records leave as one run
        uint32_t const total = warp_tot[kWarps];
        for (uint32_t at = t; at < total; at += kRouteThreads) {
            uint32_t const g = stage_at[at];
            if (g != kNone) recs[g] = stage[at];
        }
        // the next tile rewrites the shared arrays only after its first barrier
    }
}

// One CTA per slice: OR the slice's records into a shared copy of its words,
// then bulk-OR the copy into the filter in 16 KiB pieces.
constexpr uint32_t kApplyChunk = 16384;

__global__ void __launch_bounds__(kApplyThreads) k_bloom_apply(uint32_t* words, uint32_t nblocks,
                                                               unsigned long long const* recs,
                                                               uint32_t const* offsets)
{
    extern __shared__ __align__(128) uint32_t slice[];  // kSliceBlocks * 8 words
    uint32_t const sl = blockIdx.x, first = sl * kSliceBlocks;
    uint32_t const nb = nblocks - first < kSliceBlocks ? nblocks - first : kSliceBlocks;
    uint32_t const nwords = nb * 8;
    for (uint32_t i = threadIdx.x * 4; i < nwords; i += kApplyThreads * 4)
        *reinterpret_cast<uint4*>(slice + i) = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    uint32_t const beg = offsets[sl], end = offsets[sl + 1];
    for (uint32_t r = beg + threadIdx.x; r < end; r += kApplyThreads) {
        unsigned long long const rec = __ldcs(recs + r);
        uint32_t const b = uint32_t(rec >> 32), lower = uint32_t(rec);
        if (b >= nb) continue;
        // word w of block b sits at b * 8 + (w ^ swz(b)): the words that a warp
        // writes in one step spread over the banks instead of four of them
        uint32_t* blk = slice + b * 8;
        uint32_t const swz = (b >> 2) & 7u;
#pragma unroll
        for (int w = 0; w < 8; ++w) atomicOr(blk + (uint32_t(w) ^ swz), word_bit(w, lower));
    }
    __syncthreads();
    // back to the filter's word order, a block per thread
    for (uint32_t b = threadIdx.x; b < nb; b += kApplyThreads) {
        uint32_t* blk = slice + b * 8;
        uint32_t const swz = (b >> 2) & 7u;
        uint4 const lo = *reinterpret_cast<uint4 const*>(blk), hi = *reinterpret_cast<uint4 const*>(blk + 4);
        uint32_t const x[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
        uint32_t y[8];
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            uint32_t v = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) v = (uint32_t(j) == (uint32_t(w) ^ swz)) ? x[j] : v;
            y[w] = v;
        }
        *reinterpret_cast<uint4*>(blk) = make_uint4(y[0], y[1], y[2], y[3]);
        *reinterpret_cast<uint4*>(blk + 4) = make_uint4(y[4], y[5], y[6], y[7]);
    }
    fence_proxy_async();  // this thread's shared-memory writes precede the bulk reads
    __syncthreads();
    uint32_t const bytes = nwords * 4;
    if (threadIdx.x < (bytes + kApplyChunk - 1) / kApplyChunk) {
        uint32_t const off = threadIdx.x * kApplyChunk;
        uint32_t const len = bytes - off < kApplyChunk ? bytes - off : kApplyChunk;
        asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.or.b32 [%0], [%1], %2;" ::"l"(
                         words + uint64_t(first) * 8 + off / 4),
                     "r"(smem_u32(slice) + off), "r"(len)
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
}

template <int KB>
__global__ void __launch_bounds__(256) k_bloom_contains(uint32_t const* words, uint32_t nblocks, uint64_t seed,
                                                        void const* keys, uint8_t const* stencil, uint8_t* out,
                                                        uint64_t n)
{
    // kKeys keys per thread and pass, each pass's block loads issued before any
    // is tested, so a thread keeps that many random sector reads in flight
    constexpr int kKeys = 4;
    uint64_t const tile = uint64_t(blockDim.x) * kKeys;
    for (uint64_t base = uint64_t(blockIdx.x) * tile; base < n; base += uint64_t(gridDim.x) * tile) {
        uint32_t lower[kKeys];
        bool live[kKeys];
        uint4 lo[kKeys], hi[kKeys];
#pragma unroll
        for (int j = 0; j < kKeys; ++j) {
            uint64_t const i = base + uint64_t(j) * blockDim.x + threadIdx.x;
            live[j] = i < n && (!stencil || stencil[i]);
            uint32_t block = 0;
            lower[j] = 0;
            if (live[j]) locate<KB>(load_key<KB>(keys, i), seed, nblocks, block, lower[j]);
            uint4 const* p = reinterpret_cast<uint4 const*>(words + uint64_t(block) * 8);
            lo[j] = live[j] ? __ldg(p) : make_uint4(0u, 0u, 0u, 0u);
            hi[j] = live[j] ? __ldg(p + 1) : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int j = 0; j < kKeys; ++j) {
            uint64_t const i = base + uint64_t(j) * blockDim.x + threadIdx.x;
            if (i >= n) continue;
            uint32_t const w[8] = {lo[j].x, lo[j].y, lo[j].z, lo[j].w, hi[j].x, hi[j].y, hi[j].z, hi[j].w};
            bool all = live[j];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                uint32_t const bit = word_bit(k, lower[j]);
                all &= (w[k] & bit) == bit;
            }
            out[i] = all;
        }
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
    int add_mode = B2CO_BLOOM_ADD_AUTO;  // default-policy Add: see b2co_bloom_add_mode
    unsigned long long* recs = nullptr;  // partitioned Add: record workspace
    uint64_t recs_cap = 0;
    uint32_t* part = nullptr;  // partitioned Add: per-CTA slice counts, slice totals and offsets
    size_t part_words = 0;
    ScratchOrder part_order;  // the workspace serves one partitioned Add at a time
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

// B2CO_BLOOM_ADD_AUTO takes the partitioned Add for filters of at least
// kPartitionFilterBytes with batches of at least kPartitionKeysPerBlock keys per
// filter block.  Measured: on a 128 MiB filter routing ties the bulk ORs at 4
// keys per block (402 vs 412 us) and wins from 8 on (654 vs 842 us); a 2 MiB
// filter stays in L2, where the bulk ORs win at every batch size (25 vs 94 us
// at 16 keys per block) and routing's fixed cost of about 45 us dominates.
constexpr uint64_t kPartitionKeysPerBlock = 8;
constexpr uint64_t kPartitionFilterBytes = uint64_t(64) << 20;
// Keys per route-and-apply round (the record workspace holds this many).
constexpr uint64_t kPartitionRound = uint64_t(1) << 27;

template <int KB>
int launch_add_partitioned(b2co_bloom* f, void const* keys, uint8_t const* stencil, uint64_t n, cudaStream_t s)
{
    uint32_t const nblocks = uint32_t(f->num_blocks);
    uint32_t const nslices = (nblocks + kSliceBlocks - 1) / kSliceBlocks;
    uint64_t const want = n < kPartitionRound ? n : kPartitionRound;
    if (f->recs_cap < want) {
        if (f->recs) cudaFree(f->recs);
        f->recs = nullptr;
        f->recs_cap = 0;
        B2CO_CUDA(cudaMalloc(&f->recs, want * 8));
        f->recs_cap = want;
    }
    auto const route = k_bloom_route<KB>;
    auto const count = k_bloom_count<KB>;
    size_t const apply_smem = size_t(kSliceBlocks) * 32;
    size_t const rsmem = route_smem(nslices);
    B2CO_CUDA(cudaFuncSetAttribute((void const*)route, cudaFuncAttributeMaxDynamicSharedMemorySize, int(rsmem)));
    B2CO_CUDA(cudaFuncSetAttribute((void const*)k_bloom_apply, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(apply_smem)));
    int per_sm = 0;
    B2CO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (void const*)route, kRouteThreads, rsmem));
    uint32_t const route_cap = uint32_t(per_sm < 1 ? 1 : per_sm) * uint32_t(sm_count());
    // counts[route CTA][slice], then the slice totals and offsets
    size_t const part_words = size_t(route_cap) * kMaxSlices + 2 * size_t(kMaxSlices) + 1;
    if (f->part_words < part_words) {
        if (f->part) cudaFree(f->part);
        f->part = nullptr;
        f->part_words = 0;
        B2CO_CUDA(cudaMalloc(&f->part, part_words * 4));
        f->part_words = part_words;
    }
    uint32_t* counts = f->part;
    uint32_t* totals = counts + size_t(route_cap) * kMaxSlices;
    uint32_t* offsets = totals + kMaxSlices;
    if (int st = f->part_order.begin(s)) return st;
    for (uint64_t at = 0; at < n; at += kPartitionRound) {
        uint64_t const m = n - at < kPartitionRound ? n - at : kPartitionRound;
        void const* k = static_cast<char const*>(keys) + at * KB;
        uint8_t const* st = stencil ? stencil + at : nullptr;
        uint64_t const tiles = (m + kRouteTile - 1) / kRouteTile;
        uint32_t const nctas = uint32_t(tiles < route_cap ? tiles : route_cap);
        count<<<nctas, 1024, 0, s>>>(nblocks, f->seed, k, st, m, nslices, nctas, counts);
        k_bloom_colscan<<<(nslices + 255) / 256, 256, 0, s>>>(counts, nslices, nctas, totals);
        k_bloom_scan<<<1, 1024, 0, s>>>(totals, nslices, offsets);
        route<<<nctas, kRouteThreads, rsmem, s>>>(nblocks, f->seed, k, st, m, nslices, nctas, counts, offsets,
                                                      f->recs);
        k_bloom_apply<<<nslices, kApplyThreads, apply_smem, s>>>(f->words, nblocks, f->recs, offsets);
    }
    B2CO_CUDA(cudaGetLastError());
    return f->part_order.end(s);
}

int add_impl(b2co_bloom* f, void const* keys, uint8_t const* stencil, bool use_stencil, uint64_t n, cudaStream_t s)
{
    if (int st = check(f)) return st;
    if (n == 0) return B2CO_OK;
    if (!keys) return fail(B2CO_EINVAL, "BloomFilter::Add: keys must not be null when keyNum is non-zero");
    if (reinterpret_cast<uintptr_t>(keys) % f->key_bytes)
        return fail(B2CO_EINVAL, "BloomFilter::Add: keys must be aligned to the key size");
    if (use_stencil && !stencil)
        return fail(B2CO_EINVAL, "BloomFilter::AddIf: stencil must not be null when keyNum is non-zero");
    if (!f->default_policy())
        return f->key_bytes == 8 ? launch_add_policy<8>(f, keys, stencil, n, s) : launch_add_policy<4>(f, keys, stencil, n, s);
    uint64_t const nslices = (f->num_blocks + kSliceBlocks - 1) / kSliceBlocks;
    bool const part = nslices <= kMaxSlices &&
                      (f->add_mode == B2CO_BLOOM_ADD_PARTITIONED ||
                       (f->add_mode == B2CO_BLOOM_ADD_AUTO && n >= kPartitionKeysPerBlock * f->num_blocks &&
                        f->num_blocks * 32 >= kPartitionFilterBytes));
    if (part)
        return f->key_bytes == 8 ? launch_add_partitioned<8>(f, keys, stencil, n, s)
                                 : launch_add_partitioned<4>(f, keys, stencil, n, s);
    void (*k)(uint32_t*, uint32_t, uint64_t, void const*, uint8_t const*, uint64_t) = nullptr;
    if (f->add_mode != B2CO_BLOOM_ADD_ATOMIC) k = f->key_bytes == 8 ? k_bloom_add_bulk<8> : k_bloom_add_bulk<4>;
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
    if (f->recs) cudaFree(f->recs);
    if (f->part) cudaFree(f->part);
    f->part_order.release();
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
    if (mode < B2CO_BLOOM_ADD_ATOMIC || mode > B2CO_BLOOM_ADD_AUTO) return fail(B2CO_EINVAL, "unknown Add mode");
    f->add_mode = mode;
    return B2CO_OK;
}

}  // extern "C"
