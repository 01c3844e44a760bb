// noalloc.cu -- InsertAndFind (first-wins) for callers that cannot allocate.
//
// The regular first-wins InsertAndFind grows library-owned scratch with
// cudaMalloc on first use.  Some callers cannot let a library do that: a host
// application that hands all device memory to its own arena under a fixed
// budget, or a latency-critical path that must not pay for (or synchronize on)
// a device allocation in the middle of its work.  This entry point takes its
// scratch from a file-scope device array of fixed size instead, so it calls no
// cudaMalloc, no cudaFree and no allocating library routine.
//
// Costs and rules that come with the fixed array:
//  * every GPU that loads the library holds kNoAllocScratchBytes of device
//    memory for the array until the process exits;
//  * every call looks up the array's device address on the current device
//    (cudaGetSymbolAddress, which allocates nothing), so an address cached
//    across a device reset is never used; the first call on a device also
//    loads the array there, so make that first call before any stream
//    capture begins;
//  * all calls share the one array and it keeps the last call's contents:
//    calls that overlap on the GPU (other streams, other threads) race and
//    must be serialized by the caller;
//  * a batch whose scratch need exceeds the array is rejected with B2CO_ERANGE.
#include "b2co_host.h"

int b2co_oa_iaf_first_wins_on(b2co_oa_table* t, void const* pairs, void* out_found, uint8_t* out_inserted, uint64_t n,
                              uint32_t* pos, uint32_t* newbits, uint32_t* owner, bool owner_clear,
                              cudaStream_t s);

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Device address of the scratch array on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up on
// every call: a device reset reloads the module and may move the array.
int scratch_address(void** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return b2co::cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    *out = p;
    return B2CO_OK;
}

}  // namespace

extern "C" {

int b2co_oa_insert_and_find_noalloc(b2co_oa_table* t, void const* pairs, void* out_found, uint8_t* out_inserted,
                                    uint64_t n, b2co_stream stream)
{
    uint64_t capacity = 0;
    if (int st = b2co_oa_capacity(t, &capacity)) return st;
    if (n == 0 || !pairs) return B2CO_OK;
    if (!out_found || !out_inserted) return b2co::fail(B2CO_EINVAL, "InsertAndFind outputs must not be null");
    size_t const pos_bytes = align256(n * 4);
    size_t const bits_bytes = align256(((capacity + 31) / 32) * 8);  // two bitmaps of the slots
    size_t const owner_bytes = align256(capacity * 4);
    size_t const need = pos_bytes + bits_bytes + owner_bytes;
    if (n > b2co::kMaxBatch || need > kNoAllocScratchBytes)
        return b2co::fail(B2CO_ERANGE, "no-alloc InsertAndFind needs " + std::to_string(need) +
                                           " bytes of scratch (4 per item, 4 per slot, 1/4 per slot); the static "
                                           "area holds " + std::to_string(kNoAllocScratchBytes));
    void* base = nullptr;
    if (int st = scratch_address(&base)) return st;
    auto* bytes = static_cast<unsigned char*>(base);
    auto* pos = reinterpret_cast<uint32_t*>(bytes);
    auto* newbits = reinterpret_cast<uint32_t*>(bytes + pos_bytes);
    auto* owner = reinterpret_cast<uint32_t*>(bytes + pos_bytes + bits_bytes);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // the owner entries move with n inside the shared area, so they are set on every call
    if (int st = b2co_oa_iaf_first_wins_on(t, pairs, out_found, out_inserted, n, pos, newbits, owner, false, s))
        return st;
    B2CO_CUDA(cudaStreamSynchronize(s));
    return B2CO_OK;
}

}  // extern "C"
