// oa_insert.cuh -- cooperative-window kernels for the write side of the
// open-addressing containers: Insert / InsertIf, InsertOrAssign, InsertAndFind
// (race) and the placement pass of first-wins InsertAndFind.
//
// Per-key algorithm (InsertVerdict, open_addressing_ref_impl.h:489-532): walk
// the key's probe sequence bucket window by bucket window; in a window the
// first slot, in scan order, that is empty (bitwise sentinel test) or holds an
// equal key decides -- an equal key is DUPLICATE (InsertOrAssign overwrites its
// payload), an empty slot is claimed by a compare-and-swap of the whole slot
// (SUCCESS), and a lost CAS continues the scan after that slot unless the
// winner holds an equal key (DUPLICATE).  A whole cycle without a decision, or
// the empty key itself, is FAILED.
//
// B200 shape (the lookup kernels' machinery applied to writes):
//  * G lanes share a bucket window: lane r loads slots r, r+G, ... with one
//    coherent 16-byte-or-narrower load each, so a window is one or two
//    coalesced requests, not a chain of dependent slot loads;
//  * each tile keeps Q keys in flight; the tile agrees on the first deciding
//    slot by a min over shuffles, and the lane holding that slot issues the
//    CAS, whose returned value settles a lost race without another load;
//  * a key whose first window decides nothing goes to the warp's queue in
//    shared memory and is followed later, a pass of queued keys at a time, so
//    a pass waits on one window load and one CAS, never on a long probe;
//  * the window is a snapshot: slots only ever go from empty to occupied
//    during these kernels, so a slot seen occupied by another key stays so,
//    and a slot seen empty is re-checked by the CAS itself.
// Every loop is bounded by the probe cycle (and a lost CAS retries a slot a
// bounded number of times), so no kernel can spin.
#pragma once

#include "oa_kernels.cuh"

namespace b2co {

enum { kInsPlain = 0, kInsAssign = 1, kInsIafRace = 2, kInsIafPlace = 3 };

// Outputs of one insert-family launch (only the mode's fields are used).
struct InsOut {
    unsigned long long* counters;  // plain/assign: [failed, assigned] or NULL (async)
    void* found;                   // race: payload found or inserted
    uint8_t* inserted;             // race: 1 = this input inserted the key
    uint32_t* pos;                 // place: slot of every input (kNoSlot = failed)
    uint32_t* newbits;             // place: slots claimed by this batch
    uint32_t* owner;               // place: claiming input of each claimed slot (claim_bit 0 only)
    uint32_t claim_bit;            // place: flag OR-ed into pos[] of the claiming input (0 = none)
};

// Coherent window loads (L2, never a stale L1 line) with the 64-byte fill hint.
__device__ __forceinline__ uint32_t ld_win(uint32_t const* p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.L2::64B.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_win(unsigned long long const* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.L2::64B.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ U128 ld_win(U128 const* p)
{
    unsigned long long lo, hi;
    asm volatile("ld.relaxed.gpu.global.L2::64B.v2.u64 {%0, %1}, [%2];" : "=l"(lo), "=l"(hi) : "l"(p) : "memory");
    return U128{lo, hi};
}
__device__ __forceinline__ unsigned short ld_win(unsigned short const* p)
{
    unsigned short v;
    asm volatile("ld.relaxed.gpu.global.L2::64B.u16 %0, [%1];" : "=h"(v) : "l"(p) : "memory");
    return v;
}

enum { kWinOpen = 0, kWinSettled = 1, kWinIdle = 2, kWinExhausted = 3 };

// Resolution of the bucket windows of the Q keys each tile has in flight (the
// whole warp calls it; tiles whose state is not kWinOpen only take part in the
// shuffles).  On return a key's state is kWinSettled (verdict, slot and, for
// the race mode, the found payload set on every lane of the tile) or
// kWinExhausted (no slot of the window decided: probe on).  The first deciding
// slot of every key is found, then the CASes of all Q keys are issued back to
// back before any result is awaited, so a pass waits on one CAS round trip
// instead of Q.  A lost CAS updates the snapshot with the winner; a torn read
// retries the slot; a slot that keeps changing (not seen in practice) gives
// the rest of the window up after a bounded number of rounds.
template <class S, int B, int G, int Q, int ROUNDS, int MODE>
__device__ __forceinline__ void tile_insert_windows(OaArgs const& a, typename S::Raw* const (&win_base)[Q],
                                                    typename S::Raw (&w)[Q][ROUNDS], uint64_t const (&key)[Q],
                                                    uint64_t const (&val)[Q], uint32_t r, uint32_t lane0,
                                                    int (&state)[Q], int (&verdict)[Q], int (&slot)[Q],
                                                    uint64_t (&found)[Q])
{
    using Raw = typename S::Raw;
    uint32_t skip[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) skip[q] = 0;
    for (int guard = 0; guard < 4 * B + 8; ++guard) {
        bool open = false;
#pragma unroll
        for (int q = 0; q < Q; ++q) open = open || state[q] == kWinOpen;
        if (!__any_sync(0xffffffffu, open)) return;
        int s[Q], own[Q], outcome[Q];
        Raw mine[Q], old[Q];
        uint64_t got[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            own[q] = kNoStop;
            mine[q] = Raw{};
            if (state[q] == kWinOpen) {
#pragma unroll
                for (int t = ROUNDS - 1; t >= 0; --t) {
                    int const j = int(r) + t * G;
                    if (j < B && !((skip[q] >> j) & 1u)) {
                        uint64_t const k = S::key(w[q][t]);
                        if (k == a.empty_key || S::key_eq(k, key[q])) {
                            own[q] = j;
                            mine[q] = w[q][t];
                        }
                    }
                }
            }
            s[q] = own[q];
#pragma unroll
            for (int o = 1; o < G; o <<= 1) s[q] = min(s[q], __shfl_xor_sync(0xffffffffu, s[q], o));
        }
        // issue: every key's deciding lane starts its CAS (or settles a duplicate)
        Raw expected[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            outcome[q] = 0;
            got[q] = 0;
            if (state[q] == kWinOpen && s[q] != kNoStop && own[q] == s[q]) {
                Raw* sp = win_base[q] + s[q];
                if (S::key(mine[q]) != a.empty_key) {
                    outcome[q] = 2;
                    if constexpr (MODE == kInsAssign) assign_payload<S>(sp, key[q], val[q]);
                    if constexpr (MODE == kInsIafRace) got[q] = S::value(settle<S>(a, sp, mine[q]));
                } else if (!insert_expected<S>(a, mine[q], expected[q])) {
                    outcome[q] = 5;
                } else {
                    outcome[q] = -1;  // CAS in flight
                    old[q] = cas_slot(sp, expected[q], insert_desired<S>(mine[q], key[q], val[q]));
                }
            }
        }
        // settle the CASes
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (outcome[q] == -1) {
                Raw* sp = win_base[q] + s[q];
                if (raw_eq(old[q], expected[q])) {
                    outcome[q] = 1;
                    got[q] = S::is_set ? key[q] : val[q];
                } else if (S::key_eq(S::key(old[q]), key[q])) {
                    outcome[q] = 2;
                    if constexpr (MODE == kInsAssign) assign_payload<S>(sp, key[q], val[q]);
                    got[q] = S::value(old[q]);
                } else {
                    outcome[q] = S::key(old[q]) == a.empty_key ? 4 : 3;
                }
#pragma unroll
                for (int t = 0; t < ROUNDS; ++t)
                    if (int(r) + t * G == s[q]) w[q][t] = old[q];
            }
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int const src = int(lane0) + (s[q] == kNoStop ? 0 : s[q] % G);
            int const oc = __shfl_sync(0xffffffffu, outcome[q], src);
            uint64_t g = 0;
            if constexpr (MODE == kInsIafRace) g = __shfl_sync(0xffffffffu, (unsigned long long)got[q], src);
            if (state[q] == kWinOpen) {
                if (s[q] == kNoStop) {
                    state[q] = kWinExhausted;
                } else if (oc == 1 || oc == 2) {
                    state[q] = kWinSettled;
                    verdict[q] = oc == 1 ? kSuccess : kDuplicate;
                    slot[q] = s[q];
                    found[q] = g;
                } else if (oc == 5) {
                    skip[q] |= 1u << s[q];
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q)
        if (state[q] == kWinOpen) state[q] = kWinExhausted;
}

// Resident blocks per SM the write kernel is compiled for: one key per lane
// group fits 64 registers; more keys in flight keep their windows, snapshots
// and CAS operands live at once and get the registers of two blocks per SM
// instead of spilling.
#ifndef B2CO_WRITE_MINB1
#define B2CO_WRITE_MINB1 4
#endif
template <int Q>
constexpr int kWriteMinBlocks = Q == 1 ? B2CO_WRITE_MINB1 : 2;

template <class S, int B, int G, int Q, int MODE>
__global__ void __launch_bounds__(256, kWriteMinBlocks<Q>) k_insert_win(__grid_constant__ const OaArgs a, void const* pairs,
                                                       uint8_t const* stencil, uint32_t n, InsOut o)
{
    static_assert(Q <= G && G <= 8 && (G & (G - 1)) == 0, "tile shape");
    using Raw = typename S::Raw;
    constexpr int ROUNDS = (B + G - 1) / G;
    constexpr uint32_t TILES = 32 / G;
    constexpr uint32_t PASS = TILES * Q;
    static_assert(2 * PASS <= kDeferRing, "the ring must hold a pass on top of a partial one");
    constexpr uint32_t RING = kDeferRing - 1;
    __shared__ Raw qpair[8][kDeferRing];
    __shared__ uint32_t qinit[8][kDeferRing], qidx[8][kDeferRing], qpos[8][kDeferRing];

    Raw* slots = reinterpret_cast<Raw*>(a.slots);
    uint32_t const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t const r = lane % G, tile_lane0 = lane & ~uint32_t(G - 1), tile = lane / G;
    uint32_t const gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t const nwarps = (gridDim.x * blockDim.x) >> 5;
    uint32_t head = 0, count = 0;
    uint32_t failed = 0, assigned = 0;

    // The tile's first lane records a decided key.
    auto record = [&](uint32_t i, int verdict, uint32_t where, uint64_t key, uint64_t found) {
        if constexpr (MODE == kInsPlain || MODE == kInsAssign) {
            // Insert succeeds only on SUCCESS (open_addressing_ref_impl.h:282-285);
            // InsertOrAssign counts a duplicate as an assignment instead.
            failed += MODE == kInsAssign ? verdict == kFailed : verdict != kSuccess;
            assigned += verdict == kDuplicate;
        } else if constexpr (MODE == kInsIafRace) {
            Io<S>::store_payload(o.found, i, verdict == kFailed ? empty_payload<S>(a) : found);
            o.inserted[i] = verdict == kSuccess;
        } else {
            uint32_t const p = verdict == kFailed ? kNoSlot : where;
            if (verdict == kSuccess) {
                atomicOr(o.newbits + (p >> 5), 1u << (p & 31));
                if (!o.claim_bit) o.owner[p] = i;  // tables without room for the claim bit
            }
            o.pos[i] = verdict == kSuccess ? (p | o.claim_bit) : p;
        }
        (void)key;
    };
    auto enqueue = [&](bool unsettled, Raw const& pr, uint32_t init, uint32_t idx, uint32_t pos) {
        uint32_t const m = __ballot_sync(0xffffffffu, unsettled);
        if (unsettled) {
            uint32_t const e = (head + count + __popc(m & ((1u << lane) - 1u))) & RING;
            qpair[warp][e] = pr;
            qinit[warp][e] = init;
            qidx[warp][e] = idx;
            qpos[warp][e] = pos;
        }
        count += __popc(m);
    };
    // Takes up to one pass of queued keys and resolves the next window of each.
    auto follow = [&]() {
        __syncwarp();
        uint32_t const take = count < PASS ? count : PASS;
        Raw pr[Q];
        uint32_t init[Q], idx[Q], pos[Q];
        bool live[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint32_t const j = q * TILES + tile;
            live[q] = j < take;
            uint32_t const e = (head + (live[q] ? j : 0u)) & RING;
            pr[q] = qpair[warp][e];
            init[q] = qinit[warp][e];
            idx[q] = qidx[warp][e];
            pos[q] = qpos[warp][e];
        }
        __syncwarp();
        head = (head + take) & RING;
        count -= take;
        uint32_t my_step = 0;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (int(r) == q && live[q]) my_step = probe_step<S::key_bytes, B>(a.probe, S::key(pr[q]));
        Raw w[Q][ROUNDS];
        int state[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint32_t const step = __shfl_sync(0xffffffffu, my_step, tile_lane0 + q);
            state[q] = live[q] ? kWinOpen : kWinIdle;
            if (live[q]) {
                idx[q] = probe_next(idx[q], step, a.probe.capacity);
                if (idx[q] == init[q]) {  // a whole cycle: the table is full for this key
                    if (r == 0) record(pos[q], kFailed, 0, S::key(pr[q]), 0);
                    state[q] = kWinIdle;
                }
            }
            if (state[q] == kWinOpen) {
#pragma unroll
                for (int t = 0; t < ROUNDS; ++t)
                    if (int(r) + t * G < B) w[q][t] = ld_win(slots + idx[q] + r + t * G);
            }
        }
        {
            Raw* base[Q];
            uint64_t key[Q], val[Q], found[Q];
            int verdict[Q], slot[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                base[q] = slots + idx[q];
                key[q] = S::key(pr[q]);
                val[q] = S::value(pr[q]);
                verdict[q] = kFailed;
                slot[q] = 0;
                found[q] = 0;
            }
            tile_insert_windows<S, B, G, Q, ROUNDS, MODE>(a, base, w, key, val, r, tile_lane0, state, verdict, slot,
                                                          found);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                if (state[q] == kWinSettled && r == 0) record(pos[q], verdict[q], idx[q] + slot[q], key[q], found[q]);
                enqueue(state[q] == kWinExhausted && r == 0, pr[q], init[q], idx[q], pos[q]);
            }
        }
    };

    // the next pass's pairs are loaded one pass ahead (B2CO_WRITE_PREFETCH 0:
    // at the start of their own pass)
#ifndef B2CO_WRITE_PREFETCH
#define B2CO_WRITE_PREFETCH 1
#endif
    Raw nxt[Q];
    bool nin[Q];
    auto load_pass = [&](uint32_t base) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint32_t const i = base + q * TILES + tile;
            nin[q] = i < n && (!stencil || stencil[i]);
            nxt[q] = nin[q] ? Io<S>::load_pair(pairs, i) : Raw{};
        }
    };
    if (B2CO_WRITE_PREFETCH) load_pass(gwarp * PASS);
    for (uint32_t base = gwarp * PASS; base < n; base += nwarps * PASS) {
        if (!B2CO_WRITE_PREFETCH) load_pass(base);
        Raw pr[Q];
        uint32_t idx[Q];
        int state[Q];
        uint32_t my_init = 0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            pr[q] = nxt[q];
            uint64_t const key = S::key(pr[q]);
            state[q] = !nin[q] ? kWinIdle : (key == a.empty_key ? kWinSettled : kWinOpen);
            if (int(r) == q && state[q] == kWinOpen) my_init = probe_init<S::key_bytes, B>(a.probe, key);
        }
        if (B2CO_WRITE_PREFETCH) load_pass(base + nwarps * PASS);
        Raw w[Q][ROUNDS];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            idx[q] = __shfl_sync(0xffffffffu, my_init, tile_lane0 + q);
            if (state[q] == kWinOpen) {
#pragma unroll
                for (int t = 0; t < ROUNDS; ++t)
                    if (int(r) + t * G < B) w[q][t] = ld_win(slots + idx[q] + r + t * G);
            }
        }
        {
            Raw* wb[Q];
            uint64_t key[Q], val[Q], found[Q];
            int verdict[Q], slot[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                uint32_t const i = base + q * TILES + tile;
                key[q] = S::key(pr[q]);
                val[q] = S::value(pr[q]);
                wb[q] = slots + idx[q];
                verdict[q] = kFailed;
                slot[q] = 0;
                found[q] = 0;
                if (state[q] == kWinSettled) {  // the empty key itself: FAILED
                    if (r == 0) record(i, kFailed, 0, key[q], 0);
                    state[q] = kWinIdle;
                }
            }
            tile_insert_windows<S, B, G, Q, ROUNDS, MODE>(a, wb, w, key, val, r, tile_lane0, state, verdict, slot,
                                                          found);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                uint32_t const i = base + q * TILES + tile;
                if (state[q] == kWinSettled && r == 0) record(i, verdict[q], idx[q] + slot[q], key[q], found[q]);
                enqueue(state[q] == kWinExhausted && r == 0, pr[q], idx[q], idx[q], i);
            }
        }
        while (count >= PASS) follow();
    }
    while (count > 0) follow();
    if constexpr (MODE == kInsPlain || MODE == kInsAssign) {
        if (o.counters) {
            warp_add_counter(o.counters, failed);
            if (MODE == kInsAssign) warp_add_counter(o.counters + 1, assigned);
        }
    }
}

}  // namespace b2co
