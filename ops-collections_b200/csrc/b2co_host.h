// b2co_host.h -- host-side internals shared by the library's translation units:
// error reporting, launch geometry and the per-slot-layout launcher tables.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/b2co.h"
#include "b2co_common.cuh"

namespace b2co {

// Records `msg` as this thread's last error and returns `status`.
int fail(int status, std::string const& msg);
// Maps a CUDA error to B2CO_ECUDA with the failing call's name.
int cuda_fail(cudaError_t e, char const* what);
inline int ok() { return B2CO_OK; }

#define B2CO_CUDA(call)                                    \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return ::b2co::cuda_fail(e_, #call); \
    } while (0)

// Number of SMs of the current device (cached per device).
int sm_count();
// Grid for a grid-stride kernel: enough blocks for `work` items at `per_block`
// items per block, capped at the blocks that can be resident at once.
uint32_t grid_for(void const* kernel, uint32_t block, uint64_t work, uint64_t per_block);

// Orders the uses of one piece of library-owned scratch (first-wins
// InsertAndFind's, the routed Bloom Add's workspace) across the callers'
// streams: a use waits on the GPU for the previous use to end, so async calls
// on different streams cannot interleave on it.  While a stream is being
// captured into a graph nothing is added (the graph's own order holds).
struct ScratchOrder {
    cudaEvent_t done = nullptr;
    bool used = false;
    int begin(cudaStream_t s);  // before the first launch that touches the scratch
    int end(cudaStream_t s);    // after the last one
    void release();
};

// Largest batch a single launch accepts: 32-bit indices plus one grid stride
// must not overflow (the reference's CheckedBatchSize,
// detail/open_addressing/open_addressing_impl.h:534-545).
constexpr uint64_t kMaxBatch = (1ull << 32) - (1ull << 22);

// Wait policy handed to kernels that wait on asynchronous copies (limit 1 s by
// default; b2co_debug_set_wait changes it for tests).
WaitCtl wait_ctl(unsigned int* status);

// Capacity prime rule (include/utility/prime.h:15 regenerated; see runtime.cu).
uint64_t prime_at_least(uint64_t n);
uint64_t prime_table_last();

struct OaArgs;

// Lookup shape flag carried in the keys-per-lane field: scan each first window
// by 64-byte segments (B2CO_FIND_SEGMENTED in the C ABI).
constexpr uint32_t kShapeSegmented = 0x100;
// Lookup shape flag: fetch every first bucket window with one bulk (TMA) copy
// into shared memory (16-byte slots; B2CO_FIND_BULK in the C ABI).
constexpr uint32_t kShapeBulk = 0x200;
// Lookup shape flag: every warp stages its own keys (B2CO_FIND_WARP_STAGED).
constexpr uint32_t kShapeWarpStaged = 0x400;
// Lookup shape flag: warp-staged keys whose first window does not settle them
// are queued and followed a pass at a time (B2CO_FIND_DEFERRED).
constexpr uint32_t kShapeDeferred = 0x800;

// Launchers for one slot layout; B (bucket size) is dispatched at run time.
struct OaOps {
    int (*clear)(OaArgs const& a, cudaStream_t s);
    int (*insert)(OaArgs const& a, uint32_t b, void const* pairs, uint8_t const* stencil, uint32_t n, bool assign,
                  unsigned long long* counters, cudaStream_t s);
    int (*assign_if)(OaArgs const& a, uint32_t b, void const* pairs, uint8_t const* stencil, uint32_t n,
                     cudaStream_t s);
    int (*iaf_race)(OaArgs const& a, uint32_t b, void const* pairs, void* found, uint8_t* inserted, uint32_t n,
                    cudaStream_t s);
    int (*iaf_first)(OaArgs const& a, uint32_t b, void const* pairs, void* found, uint8_t* inserted, uint32_t n,
                     uint32_t* pos, uint32_t* newbits, uint32_t* owner, cudaStream_t s);
    int (*find)(OaArgs const& a, uint32_t b, uint32_t lanes, uint32_t items, bool contains, void const* keys,
                uint8_t const* stencil, void* out, uint32_t n, WaitCtl wc, cudaStream_t s);
    int (*erase)(OaArgs const& a, uint32_t b, void const* keys, uint32_t n, unsigned long long* counters,
                 cudaStream_t s);
    int (*count)(OaArgs const& a, uint32_t b, void const* keys, uint32_t n, unsigned long long* counter,
                 cudaStream_t s);
};

extern OaOps const kOpsSet4, kOpsSet8, kOpsMap44, kOpsMap48, kOpsMap84, kOpsMap88;
// 2-byte-key layouts (integer and fp16 keys) and the floating-point-key layouts.
extern OaOps const kOpsSet2, kOpsMap22, kOpsSet2F, kOpsMap22F, kOpsSet4F, kOpsMap44F, kOpsMap48F, kOpsSet8F,
    kOpsMap84F, kOpsMap88F;

// Launchers of a layout (nullptr for combinations without one).
OaOps const* oa_ops_for(uint32_t key_bytes, uint32_t value_bytes, uint32_t key_kind);
// Bytes of one slot: Pair<K,V> aligned to min(16, bitceil(sizeof K + sizeof V)),
// the payload at the next offset aligned to its size (pair.inl:19-24), or a bare key.
uint32_t oa_slot_bytes(uint32_t key_bytes, uint32_t value_bytes);

struct GroupArgs;

// Launchers of the persistent group kernels for one slot layout.
struct GroupOps {
    // shape: lanes | keys per lane group << 8 | threads per block << 16
    int (*find)(GroupArgs const& g, uint32_t b, uint32_t shape, bool contains, void const* keys, void* out,
                uint64_t n, cudaStream_t s);
    int (*insert)(GroupArgs const& g, uint32_t b, void const* pairs, uint64_t n, unsigned long long* failed,
                  cudaStream_t s);
};

extern GroupOps const kGroupSet4, kGroupSet8, kGroupMap44, kGroupMap48, kGroupMap84, kGroupMap88;

}  // namespace b2co
