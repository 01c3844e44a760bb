// b2co_common.cuh -- primitives shared by every B200 kernel of the
// bulk-container library: the public hashing / probing / slot primitives
// (include/b2co/device.cuh) plus the library-internal device helpers (slot
// CAS, read-only and coherent slot loads, TMA bulk copies and mbarriers with
// bounded waits).
#pragma once

#include "../../include/b2co/device.cuh"

namespace b2co {

// Device-side wait policy of kernels that wait on asynchronous copies: a wait
// that exceeds `ns` nanoseconds stores kStatusTimeout into *status and the
// kernel returns instead of waiting on.
constexpr unsigned int kStatusTimeout = 1;
struct WaitCtl {
    unsigned int* status;
    unsigned long long ns;
    unsigned int probe_timeout;  // test hook: the first wait is on a barrier nothing arrives on
};

#ifdef __CUDACC__
// Atomic compare-and-swap of a whole slot: 32-, 64- or 128-bit (the 128-bit form
// needs sm_90+; it publishes key and payload together, so no reader ever sees a
// key without its payload).
// 2-byte slots (the narrow CAS of open_addressing_ref_impl.h:187-199) use the
// native 16-bit compare-and-swap of sm_70+.
__device__ __forceinline__ unsigned short cas_slot(unsigned short* p, unsigned short e, unsigned short d)
{
    return atomicCAS(p, e, d);
}
__device__ __forceinline__ uint32_t cas_slot(uint32_t* p, uint32_t e, uint32_t d) { return atomicCAS(p, e, d); }
__device__ __forceinline__ unsigned long long cas_slot(unsigned long long* p, unsigned long long e,
                                                       unsigned long long d)
{
    return atomicCAS(p, e, d);
}
__device__ __forceinline__ U128 cas_slot(U128* p, U128 e, U128 d) { return atomicCAS(p, e, d); }

// Read-only (non-coherent) loads for kernels that never write the table, with
// an L2 prefetch-size hint (B2CO_RO_FILL bytes: 64 by default, 0 for none): a
// bucket window is a random 80-byte read, and larger fills only bring in
// neighbouring slots no query of this launch is likely to touch.
#ifndef B2CO_RO_FILL
#define B2CO_RO_FILL 64
#endif
#if B2CO_RO_FILL == 0
#define B2CO_LD_RO "ld.global.nc"
#elif B2CO_RO_FILL == 64
#define B2CO_LD_RO "ld.global.nc.L2::64B"
#elif B2CO_RO_FILL == 128
#define B2CO_LD_RO "ld.global.nc.L2::128B"
#elif B2CO_RO_FILL == 256
#define B2CO_LD_RO "ld.global.nc.L2::256B"
#else
#error "B2CO_RO_FILL must be 0, 64, 128 or 256"
#endif
__device__ __forceinline__ unsigned short ld_ro(unsigned short const* p)
{
    unsigned short v;
    asm(B2CO_LD_RO ".u16 %0, [%1];" : "=h"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ uint32_t ld_ro(uint32_t const* p)
{
    uint32_t v;
    asm(B2CO_LD_RO ".u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned long long ld_ro(unsigned long long const* p)
{
    unsigned long long v;
    asm(B2CO_LD_RO ".u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ U128 ld_ro(U128 const* p)
{
    unsigned long long lo, hi;
    asm(B2CO_LD_RO ".v2.u64 {%0, %1}, [%2];" : "=l"(lo), "=l"(hi) : "l"(p));
    return U128{lo, hi};
}
// ---- bulk copies (TMA, untiled) and mbarriers --------------------------------
__device__ __forceinline__ uint32_t smem_u32(void const* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Orders this thread's generic-proxy shared-memory accesses before later async-proxy (bulk copy) ones.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Global -> shared bulk copy completing on `bar`; dst, src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, void const* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Waits for phase `parity` of `bar` for at most `limit_ns` nanoseconds.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t const t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

// Coherent loads for kernels that race with writers to the same table.
__device__ __forceinline__ unsigned short ld_rw(unsigned short const* p)
{
    return *reinterpret_cast<volatile unsigned short const*>(p);
}
__device__ __forceinline__ uint32_t ld_rw(uint32_t const* p) { return *reinterpret_cast<volatile uint32_t const*>(p); }
__device__ __forceinline__ unsigned long long ld_rw(unsigned long long const* p)
{
    return *reinterpret_cast<volatile unsigned long long const*>(p);
}
__device__ __forceinline__ U128 ld_rw(U128 const* p)
{
    unsigned long long lo, hi;
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(lo), "=l"(hi) : "l"(p) : "memory");
    return U128{lo, hi};
}
#endif

}  // namespace b2co
