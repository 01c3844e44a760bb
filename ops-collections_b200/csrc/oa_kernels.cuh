// oa_kernels.cuh -- sm_100a kernels for the open-addressing containers
// (StaticMap / StaticSet / DynamicMap submaps).
//
// Per-key algorithms restate detail/open_addressing/open_addressing_ref_impl.h:
// probe bucket windows from the scheme's start index; inside a window scan the
// slots in order; an empty-key slot ends a lookup (or is claimed by an insert),
// an equal key is a hit/duplicate; a full cycle of the probe sequence fails.
//
// B200 design:
//  * a slot is published with ONE atomic CAS of the whole slot (32/64/128-bit),
//    so the key and payload appear together and no reader ever waits for a
//    payload (the reference's unbounded WaitForPayload spin does not exist);
//  * lookups read the table through the non-coherent path with 16-byte vector
//    loads and a 64-byte L2 fill hint.  The default lookup (k_find_wdefer)
//    stages keys per warp with bulk copies, gives each bucket window G lanes
//    (one slot per lane and round, the tile agreeing on the first stopping
//    slot by a min over shuffles), and queues the rare keys that need further
//    windows so each pass waits on one window load; one-lane-per-key and
//    ballot-resolved shapes remain selectable;
//  * every loop is bounded by the probe cycle, so no kernel can spin.
#pragma once

#include <cstdint>
#include <type_traits>

#include "b2co_common.cuh"

namespace b2co {

constexpr uint32_t kNoSlot = 0xffffffffu;

struct OaArgs {
    void* slots;
    ProbeParams probe;
    uint64_t empty_key;
    uint64_t empty_value;
    uint64_t erased_key;
    uint32_t write_shape;  // insert-family kernel shape: 0 = default, else (lanes << 8) | keys per tile
};

template <int N>
using WordT = typename std::conditional<N == 8, unsigned long long,
              typename std::conditional<N == 2, unsigned short, uint32_t>::type>::type;

template <class S>
struct Io {
    static constexpr int PB = S::is_set ? S::key_bytes : S::value_bytes;  // payload bytes
    using Key = WordT<S::key_bytes>;
    using Payload = WordT<PB>;
    using Raw = typename S::Raw;
    __device__ static uint64_t load_key(void const* keys, uint32_t i)
    {
        return uint64_t(__ldg(reinterpret_cast<Key const*>(keys) + i));
    }
    __device__ static void store_payload(void* out, uint32_t i, uint64_t v)
    {
        reinterpret_cast<Payload*>(out)[i] = Payload(v);
    }
    __device__ static Raw load_pair(void const* pairs, uint32_t i) { return ld_ro(reinterpret_cast<Raw const*>(pairs) + i); }
};

template <class S>
__device__ __forceinline__ uint64_t empty_payload(OaArgs const& a)
{
    return S::is_set ? a.empty_key : a.empty_value;
}

// The slot to CAS an insert against.  Slots up to 8 bytes compare the whole
// canonical empty pair (PackCas, open_addressing_ref_impl.h:126-147); 16-byte
// slots compare the key only (CasDependentWrite, :164-185), which here means
// "the slot exactly as loaded, whose key was seen empty".
template <class S>
__device__ __forceinline__ bool insert_expected(OaArgs const& a, typename S::Raw cur, typename S::Raw& expected)
{
    if constexpr (S::bytes == 16) {
        expected = cur;
        return true;
    } else {
        expected = S::make(a.empty_key, a.empty_value);
        return raw_eq(cur, expected);
    }
}

// The slot written by an insert: key and payload, the rest of the slot kept.
template <class S>
__device__ __forceinline__ typename S::Raw insert_desired(typename S::Raw cur, uint64_t k, uint64_t v)
{
    if constexpr (S::bytes == 16) {
        U128 r = cur;
        r.lo = (r.lo & ~S::kmask) | (k & S::kmask);
        if constexpr (S::value_offset == 8) r.hi = (r.hi & ~S::vmask) | (v & S::vmask);
        return r;
    } else {
        return S::make(k, v);
    }
}

// Payload store of an existing key (AssignPayload, open_addressing_ref_impl.h:208-220):
// a whole-slot store for slots up to 8 bytes, the payload field (at byte 8)
// of a 16-byte slot otherwise.
template <class S>
__device__ __forceinline__ void assign_payload(typename S::Raw* slot, uint64_t k, uint64_t v)
{
    if constexpr (S::is_set) {
        return;
    } else if constexpr (S::bytes <= 8) {
        *reinterpret_cast<volatile typename S::Raw*>(slot) = S::make(k, v);
    } else if constexpr (S::value_bytes == 8) {
        reinterpret_cast<volatile unsigned long long*>(slot)[1] = v;
    } else if constexpr (S::value_bytes == 4) {
        reinterpret_cast<volatile uint32_t*>(slot)[2] = uint32_t(v);
    } else {
        reinterpret_cast<volatile unsigned short*>(slot)[4] = (unsigned short)v;
    }
}

// A 16-byte slot seen through a plain vector load could in principle be torn
// against a concurrent 128-bit CAS.  Only a key-matching slot whose payload
// still reads as the empty payload is ambiguous; re-read it atomically.
template <class S>
__device__ __forceinline__ typename S::Raw settle(OaArgs const& a, typename S::Raw* slot, typename S::Raw cur)
{
    if constexpr (S::bytes == 16 && !S::is_set) {
        if (S::value(cur) == (a.empty_value & S::vmask)) return cas_slot(slot, cur, cur);
    }
    return cur;
}

// ----------------------------------------------------------------------------
// Insert / InsertIf / InsertOrAssign
// (InsertVerdict, open_addressing_ref_impl.h:489-532; kernels.h:46-182)
// ----------------------------------------------------------------------------

enum { kFailed = 0, kSuccess = 1, kDuplicate = 2 };

template <class S, int B, bool ASSIGN>
__device__ __forceinline__ int insert_one(OaArgs const& a, uint64_t key, uint64_t val)
{
    using Raw = typename S::Raw;
    if (key == a.empty_key) return kFailed;
    Raw* slots = reinterpret_cast<Raw*>(a.slots);
    uint32_t const init = probe_init<S::key_bytes, B>(a.probe, key);
    uint32_t idx = init, step = 0;
    for (;;) {
#pragma unroll
        for (int j = 0; j < B; ++j) {
            Raw* sp = slots + idx + j;
            Raw cur = ld_rw(sp);
            uint64_t k = S::key(cur);
            if (S::key_eq(k, key)) {
                if constexpr (ASSIGN) assign_payload<S>(sp, key, val);
                return kDuplicate;
            }
            if (k == a.empty_key) {
                Raw expected;
                if (!insert_expected<S>(a, cur, expected)) continue;
                Raw old = cas_slot(sp, expected, insert_desired<S>(cur, key, val));
                if (raw_eq(old, expected)) return kSuccess;
                if (S::key_eq(S::key(old), key)) {
                    if constexpr (ASSIGN) assign_payload<S>(sp, key, val);
                    return kDuplicate;
                }
            }
        }
        if (step == 0) step = probe_step<S::key_bytes, B>(a.probe, key);
        idx = probe_next(idx, step, a.probe.capacity);
        if (idx == init) return kFailed;
    }
}

__device__ __forceinline__ void warp_add_counter(unsigned long long* counter, uint32_t v)
{
    uint32_t sum = __reduce_add_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(counter, (unsigned long long)sum);
}

// counters[0] += failed, counters[1] += assigned (NULL counters = async form).
template <class S, int B, bool ASSIGN>
__global__ void __launch_bounds__(256) k_insert(__grid_constant__ const OaArgs a, void const* pairs, uint8_t const* stencil, uint32_t n,
                                                unsigned long long* counters)
{
    uint32_t failed = 0, assigned = 0;
    uint32_t const stride = gridDim.x * blockDim.x;
    // warp-uniform trip count so the counter reduction sees every lane
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        uint32_t i = base + (threadIdx.x & 31);
        if (i < n && (!stencil || stencil[i])) {
            typename S::Raw p = Io<S>::load_pair(pairs, i);
            int r = insert_one<S, B, ASSIGN>(a, S::key(p), S::value(p));
            // Insert succeeds only on SUCCESS (open_addressing_ref_impl.h:282-285), so a
            // duplicate is a failure; InsertOrAssign counts it as an assignment instead.
            failed += ASSIGN ? r == kFailed : r != kSuccess;
            assigned += r == kDuplicate;
        }
    }
    if (counters) {
        warp_add_counter(counters, failed);
        if (ASSIGN) warp_add_counter(counters + 1, assigned);
    }
}

// AssignIf (Assign, open_addressing_ref_impl.h:384-410): payload overwrite of
// existing keys only; an empty slot ends the search.
template <class S, int B>
__global__ void __launch_bounds__(256) k_assign_if(__grid_constant__ const OaArgs a, void const* pairs, uint8_t const* stencil, uint32_t n)
{
    using Raw = typename S::Raw;
    Raw* slots = reinterpret_cast<Raw*>(a.slots);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (stencil && !stencil[i]) continue;
        Raw p = Io<S>::load_pair(pairs, i);
        uint64_t key = S::key(p);
        uint32_t const init = probe_init<S::key_bytes, B>(a.probe, key);
        uint32_t idx = init, step = 0;
        bool done = false;
        while (!done) {
#pragma unroll
            for (int j = 0; j < B; ++j) {
                if (done) break;
                Raw* sp = slots + idx + j;
                uint64_t k = S::key(ld_rw(sp));
                if (k == a.empty_key) done = true;
                else if (S::key_eq(k, key)) {
                    assign_payload<S>(sp, key, S::value(p));
                    done = true;
                }
            }
            if (done) break;
            if (step == 0) step = probe_step<S::key_bytes, B>(a.probe, key);
            idx = probe_next(idx, step, a.probe.capacity);
            if (idx == init) break;
        }
    }
}

// ----------------------------------------------------------------------------
// InsertAndFind, race mode: exactly the reference's concurrent semantics
// (open_addressing_ref_impl.h:301-330, 543-565); duplicates in one batch race.
// ----------------------------------------------------------------------------

template <class S, int B>
__global__ void __launch_bounds__(256) k_iaf_race(__grid_constant__ const OaArgs a, void const* pairs, void* out_found,
                                                  uint8_t* out_inserted, uint32_t n)
{
    using Raw = typename S::Raw;
    Raw* slots = reinterpret_cast<Raw*>(a.slots);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Raw p = Io<S>::load_pair(pairs, i);
        uint64_t key = S::key(p), val = S::value(p);
        uint64_t found = empty_payload<S>(a);
        uint8_t inserted = 0;
        if (key != a.empty_key) {
            uint32_t const init = probe_init<S::key_bytes, B>(a.probe, key);
            uint32_t idx = init, step = 0;
            bool done = false;
            while (!done) {
#pragma unroll
                for (int j = 0; j < B; ++j) {
                    if (done) break;
                    Raw* sp = slots + idx + j;
                    Raw cur = ld_rw(sp);
                    uint64_t k = S::key(cur);
                    if (S::key_eq(k, key)) {
                        found = S::value(settle<S>(a, sp, cur));
                        done = true;
                    } else if (k == a.empty_key) {
                        Raw expected;
                        if (!insert_expected<S>(a, cur, expected)) continue;
                        Raw old = cas_slot(sp, expected, insert_desired<S>(cur, key, val));
                        if (raw_eq(old, expected)) {
                            found = S::is_set ? key : val;
                            inserted = 1;
                            done = true;
                        } else if (S::key_eq(S::key(old), key)) {
                            found = S::value(old);
                            done = true;
                        }
                    }
                }
                if (done) break;
                if (step == 0) step = probe_step<S::key_bytes, B>(a.probe, key);
                idx = probe_next(idx, step, a.probe.capacity);
                if (idx == init) break;
            }
        }
        Io<S>::store_payload(out_found, i, found);
        out_inserted[i] = inserted;
    }
}

// ----------------------------------------------------------------------------
// InsertAndFind, first-wins mode: deterministic, equal to inserting the batch
// sequentially in input order (the golden of tests/common/golden.h:104-131).
// When the table has fewer than 2^31 slots, pos[i] of the input that claimed a
// slot carries kClaimBit, and owner[] (one entry per slot) holds kNoOwner
// between batches:
//   place   : every key finds or claims its slot; pos[i] = slot; a claimer
//             marks the slot in `newbits` (claimed by this batch) and writes
//             nothing else -- a unique key costs no random access besides its
//             window and its CAS;
//   min     : the other inputs on a claimed slot lower owner[slot] to the
//             least of their indices (atomicMin); the first of them marks the
//             slot in `dup`;
//   claim   : the claimer of a slot in `dup` lowers owner[slot] to its own
//             index when smaller;
//   final   : a claimer whose slot is not in `dup` is the inserted input (its
//             CAS stored its pair); on a slot in `dup` the input owner[slot]
//             names is the inserted one, every input there finds that input's
//             payload (read from the inputs, never a racing slot), and an owner
//             that was not the claimer rewrites the payload; inputs on older
//             slots find the stored payload;
//   restore : the claimers of slots in `dup` put owner[slot] back to kNoOwner.
// Tables of 2^31 slots or more have no room for the claim bit in pos[]: there
// the claimer writes owner[slot] in place, min lowers it over every input on
// the slot, final reads it for all of them, and claim and restore do not run.
// `dup` is the bitmap right after `newbits` (both cleared before place).
// ----------------------------------------------------------------------------

constexpr uint32_t kClaimBit = 0x80000000u;
constexpr uint32_t kNoOwner = 0xffffffffu;

template <class S, int B>
__global__ void __launch_bounds__(256) k_iaf_place(__grid_constant__ const OaArgs a, void const* pairs, uint32_t n, uint32_t* pos,
                                                   uint32_t* newbits, uint32_t* owner, uint32_t claim_bit)
{
    using Raw = typename S::Raw;
    Raw* slots = reinterpret_cast<Raw*>(a.slots);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Raw p = Io<S>::load_pair(pairs, i);
        uint64_t key = S::key(p), val = S::value(p);
        uint32_t where = kNoSlot;
        if (key != a.empty_key) {
            uint32_t const init = probe_init<S::key_bytes, B>(a.probe, key);
            uint32_t idx = init, step = 0;
            bool done = false;
            while (!done) {
#pragma unroll
                for (int j = 0; j < B; ++j) {
                    if (done) break;
                    Raw* sp = slots + idx + j;
                    Raw cur = ld_rw(sp);
                    uint64_t k = S::key(cur);
                    if (S::key_eq(k, key)) {
                        where = idx + j;
                        done = true;
                    } else if (k == a.empty_key) {
                        Raw expected;
                        if (!insert_expected<S>(a, cur, expected)) continue;
                        Raw old = cas_slot(sp, expected, insert_desired<S>(cur, key, val));
                        if (raw_eq(old, expected)) {
                            where = idx + j;
                            atomicOr(newbits + (where >> 5), 1u << (where & 31));
                            if (!claim_bit) owner[where] = i;
                            where |= claim_bit;
                            done = true;
                        } else if (S::key_eq(S::key(old), key)) {
                            where = idx + j;
                            done = true;
                        }
                    }
                }
                if (done) break;
                if (step == 0) step = probe_step<S::key_bytes, B>(a.probe, key);
                idx = probe_next(idx, step, a.probe.capacity);
                if (idx == init) break;
            }
        }
        pos[i] = where;
    }
}

__device__ __forceinline__ bool bit_set(uint32_t const* bits, uint32_t s) { return (bits[s >> 5] >> (s & 31)) & 1u; }

// The passes after placement take four inputs a thread: one 16-byte load of
// their pos[] entries, then each dependent step (bitmap word, owner entry,
// input pair) issued for all four before any is used, so a thread keeps four
// independent chains of loads in flight.
constexpr uint32_t kIafItems = 4;

__device__ __forceinline__ void load_pos4(uint32_t const* pos, uint32_t n, uint32_t i0, uint32_t (&p)[kIafItems])
{
    if (i0 + kIafItems <= n) {
        uint4 const v = __ldcs(reinterpret_cast<uint4 const*>(pos + i0));  // pos[] is 16-byte aligned
        p[0] = v.x, p[1] = v.y, p[2] = v.z, p[3] = v.w;
    } else {
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k) p[k] = i0 + k < n ? pos[i0 + k] : kNoSlot;
    }
}

__device__ __forceinline__ bool bit_of(uint32_t word, uint32_t s) { return (word >> (s & 31)) & 1u; }

template <class S>  // one copy per slot layout's translation unit
__global__ void __launch_bounds__(256) k_iaf_min(uint32_t const* pos, uint32_t const* newbits, uint32_t* dup,
                                                 uint32_t* owner, uint32_t n, uint32_t claim_bit)
{
    uint32_t const groups = (n + kIafItems - 1) / kIafItems;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
        uint32_t const i0 = q * kIafItems;
        uint32_t p[kIafItems], w[kIafItems];
        load_pos4(pos, n, i0, p);
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k)  // failed inputs and the claimers themselves skip
            w[k] = p[k] != kNoSlot && !(p[k] & claim_bit) ? newbits[(p[k] & ~claim_bit) >> 5] : 0u;
        uint32_t was[kIafItems];
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k) {
            uint32_t const sl = p[k] & ~claim_bit;
            was[k] = w[k] && bit_of(w[k], sl) ? atomicMin(owner + sl, i0 + k) : 0u;
        }
        if (claim_bit) {
#pragma unroll
            for (uint32_t k = 0; k < kIafItems; ++k) {
                uint32_t const sl = p[k] & ~claim_bit;
                if (w[k] && bit_of(w[k], sl) && was[k] == kNoOwner) atomicOr(dup + (sl >> 5), 1u << (sl & 31));
            }
        }
    }
}

// The claimer of a slot in `dup` is the only writer of its owner entry in this
// launch.
template <class S>
__global__ void __launch_bounds__(256) k_iaf_claim(uint32_t const* pos, uint32_t const* dup, uint32_t* owner,
                                                   uint32_t n, uint32_t claim_bit)
{
    uint32_t const groups = (n + kIafItems - 1) / kIafItems;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
        uint32_t const i0 = q * kIafItems;
        uint32_t p[kIafItems], w[kIafItems], o[kIafItems];
        load_pos4(pos, n, i0, p);
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k)
            w[k] = p[k] != kNoSlot && (p[k] & claim_bit) ? dup[(p[k] & ~claim_bit) >> 5] : 0u;
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k)
            o[k] = w[k] && bit_of(w[k], p[k] & ~claim_bit) ? owner[p[k] & ~claim_bit] : 0u;
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k)
            if (w[k] && bit_of(w[k], p[k] & ~claim_bit) && i0 + k < o[k]) owner[p[k] & ~claim_bit] = i0 + k;
    }
}

// Puts owner[] back to all-ones on the slots in `dup` (batches small against
// the table; a large one clears the whole array instead).
template <class S>
__global__ void __launch_bounds__(256) k_iaf_restore(uint32_t const* pos, uint32_t const* dup, uint32_t* owner,
                                                     uint32_t n, uint32_t claim_bit)
{
    uint32_t const groups = (n + kIafItems - 1) / kIafItems;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
        uint32_t const i0 = q * kIafItems;
        uint32_t p[kIafItems], w[kIafItems];
        load_pos4(pos, n, i0, p);
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k)
            w[k] = p[k] != kNoSlot && (p[k] & claim_bit) ? dup[(p[k] & ~claim_bit) >> 5] : 0u;
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k)
            if (w[k] && bit_of(w[k], p[k] & ~claim_bit)) owner[p[k] & ~claim_bit] = kNoOwner;
    }
}

template <class S>
__global__ void __launch_bounds__(256) k_iaf_final(__grid_constant__ const OaArgs a, void const* pairs, uint32_t const* pos,
                                                   uint32_t const* newbits, uint32_t const* dup,
                                                   uint32_t const* owner, void* out_found, uint8_t* out_inserted,
                                                   uint32_t n, uint32_t claim_bit)
{
    using Raw = typename S::Raw;
    Raw* slots = reinterpret_cast<Raw*>(a.slots);
    enum : uint32_t { kNone, kAlone, kShared, kOld };
    uint32_t const groups = (n + kIafItems - 1) / kIafItems;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
        uint32_t const i0 = q * kIafItems;
        uint32_t p[kIafItems], w[kIafItems], kind[kIafItems], m[kIafItems];
        load_pos4(pos, n, i0, p);
        // a claimer reads its dup bit, any other input the claimed bit of its slot
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k) {
            uint32_t const sl = p[k] & ~claim_bit;
            w[k] = p[k] == kNoSlot ? 0u : (p[k] & claim_bit) ? dup[sl >> 5] : newbits[sl >> 5];
        }
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k) {
            uint32_t const sl = p[k] & ~claim_bit;
            bool const claimed = p[k] != kNoSlot && (p[k] & claim_bit);
            // a claimer alone on its slot: its CAS stored its pair.  Otherwise a
            // slot claimed by this batch names its inserted input in owner[]
            // (claimers reach this only through dup), and an older slot holds
            // the payload to find.
            kind[k] = p[k] == kNoSlot ? kNone
                      : claimed       ? (bit_of(w[k], sl) ? kShared : kAlone)
                                      : (bit_of(w[k], sl) ? kShared : kOld);
        }
        Raw v[kIafItems];
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k) {
            uint32_t const sl = p[k] & ~claim_bit;
            m[k] = kind[k] == kShared ? owner[sl] : i0 + k;
            if (kind[k] == kOld) v[k] = ld_rw(slots + sl);
        }
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k)
            if (kind[k] == kAlone || kind[k] == kShared) v[k] = Io<S>::load_pair(pairs, m[k]);
#pragma unroll
        for (uint32_t k = 0; k < kIafItems; ++k) {
            uint32_t const i = i0 + k;
            if (i >= n) break;
            uint64_t found = empty_payload<S>(a);
            uint8_t inserted = 0;
            if (kind[k] != kNone) {
                found = S::value(v[k]);
                if (kind[k] == kAlone || (kind[k] == kShared && m[k] == i)) {
                    inserted = 1;
                    // an owner that is not the claimer rewrites the payload
                    if (kind[k] == kShared && !(p[k] & claim_bit))
                        assign_payload<S>(slots + (p[k] & ~claim_bit), S::key(v[k]), found);
                }
            }
            Io<S>::store_payload(out_found, i, found);
            out_inserted[i] = inserted;
        }
    }
}

// ----------------------------------------------------------------------------
// Find / Contains (FindAndContains, open_addressing_ref_impl.h:567-605)
// ----------------------------------------------------------------------------

// Whether a loaded window holds a slot that ends the scan (empty or equal); the
// first such slot is copied into `stop`.  The copy is an unrolled select, so the
// window stays in registers (indexing it with a computed slot number would move
// it to local memory).
template <class S, int B>
__device__ __forceinline__ bool scan_window(typename S::Raw const (&w)[B], uint64_t key, uint64_t empty_key,
                                            typename S::Raw& stop)
{
    bool found = false;
#pragma unroll
    for (int j = B - 1; j >= 0; --j) {
        uint64_t k = S::key(w[j]);
        if (k == empty_key || S::key_eq(k, key)) {
            stop = w[j];
            found = true;
        }
    }
    return found;
}

template <class S, int B>
__device__ __forceinline__ void load_window(typename S::Raw const* slots, uint32_t idx, typename S::Raw (&w)[B])
{
#pragma unroll
    for (int j = 0; j < B; ++j) w[j] = ld_ro(slots + idx + j);
}

// Continue a lookup whose first window held neither the key nor an empty slot.
template <class S, int B>
__device__ __noinline__ bool find_rest(OaArgs const& a, uint64_t key, uint32_t init, uint64_t& payload)
{
    using Raw = typename S::Raw;
    Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
    uint32_t const step = probe_step<S::key_bytes, B>(a.probe, key);
    uint32_t idx = probe_next(init, step, a.probe.capacity);
    while (idx != init) {
        Raw w[B];
        load_window<S, B>(slots, idx, w);
        Raw stop;
        if (scan_window<S, B>(w, key, a.empty_key, stop)) {
            bool hit = S::key(stop) != a.empty_key;  // an empty slot ends the scan first
            payload = hit ? S::value(stop) : empty_payload<S>(a);
            return hit;
        }
        idx = probe_next(idx, step, a.probe.capacity);
    }
    payload = empty_payload<S>(a);
    return false;
}

// One lane per key, ITEMS keys per lane in flight: all windows are loaded
// before any is resolved, so a lane keeps ITEMS * B independent loads open.
template <class S, int B, int ITEMS, bool CONTAINS>
__global__ void __launch_bounds__(256) k_find_lane(__grid_constant__ const OaArgs a, void const* keys, uint8_t const* stencil, void* out,
                                                   uint32_t n)
{
    using Raw = typename S::Raw;
    Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
    uint32_t const stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += stride * ITEMS) {
        uint64_t key[ITEMS];
        uint32_t init[ITEMS];
        bool live[ITEMS];
        Raw w[ITEMS][B];
#pragma unroll
        for (int t = 0; t < ITEMS; ++t) {
            uint32_t i = base + t * stride;
            live[t] = i < n && (!stencil || stencil[i]);
            key[t] = live[t] ? Io<S>::load_key(keys, i) : 0;
            init[t] = live[t] ? probe_init<S::key_bytes, B>(a.probe, key[t]) : 0;
        }
#pragma unroll
        for (int t = 0; t < ITEMS; ++t)
            if (live[t]) load_window<S, B>(slots, init[t], w[t]);
#pragma unroll
        for (int t = 0; t < ITEMS; ++t) {
            uint32_t i = base + t * stride;
            if (i >= n) continue;
            uint64_t payload = empty_payload<S>(a);
            bool hit = false;
            if (live[t]) {
                Raw stop;
                if (scan_window<S, B>(w[t], key[t], a.empty_key, stop)) {
                    hit = S::key(stop) != a.empty_key;
                    if (hit) payload = S::value(stop);
                } else {
                    hit = find_rest<S, B>(a, key[t], init[t], payload);
                }
            }
            if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = hit;
            else Io<S>::store_payload(out, i, payload);
        }
    }
}

// G lanes per key: lane r of a tile loads slots r, r+G, ... of the window; the
// tile resolves the window with one ballot pair per round and the lane holding
// the hit slot hands its payload to the tile's first lane, which writes it.
template <class S, int B, int G, bool CONTAINS>
__global__ void __launch_bounds__(256) k_find_tile(__grid_constant__ const OaArgs a, void const* keys, uint8_t const* stencil, void* out,
                                                   uint32_t n)
{
    using Raw = typename S::Raw;
    constexpr int ROUNDS = (B + G - 1) / G;
    constexpr uint32_t TILES = 32 / G;
    constexpr uint32_t TILE_MASK = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
    Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
    uint32_t const lane = threadIdx.x & 31, r = lane % G, tile_shift = (lane / G) * G;
    uint32_t const warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * TILES; base < n; base += warps * TILES) {
        uint32_t const i = base + lane / G;
        bool const live = i < n && (!stencil || stencil[i]);
        uint64_t const key = live ? Io<S>::load_key(keys, i) : 0;
        uint32_t const init = live ? probe_init<S::key_bytes, B>(a.probe, key) : 0;
        uint32_t idx = init, step = 0;
        bool done = !live, hit = false;
        int stop_j = -1;
        uint64_t payload = empty_payload<S>(a);
        while (__any_sync(0xffffffffu, !done)) {
            uint32_t stop_bits = 0, hit_bits = 0;
            Raw w[ROUNDS];
#pragma unroll
            for (int t = 0; t < ROUNDS; ++t) {
                int j = int(r) + t * G;
                bool own = !done && j < B;
                uint64_t k = 0;
                if (own) {
                    w[t] = ld_ro(slots + idx + j);
                    k = S::key(w[t]);
                }
                bool is_hit = own && S::key_eq(k, key) && k != a.empty_key;
                bool is_stop = own && (k == a.empty_key || is_hit);
                stop_bits |= ((__ballot_sync(0xffffffffu, is_stop) >> tile_shift) & TILE_MASK) << (t * G);
                hit_bits |= ((__ballot_sync(0xffffffffu, is_hit) >> tile_shift) & TILE_MASK) << (t * G);
            }
            if (!done) {
                if (stop_bits) {
                    stop_j = __ffs(stop_bits) - 1;
                    hit = (hit_bits >> stop_j) & 1u;
                    done = true;
                    if (hit) {
#pragma unroll
                        for (int t = 0; t < ROUNDS; ++t)
                            if (int(r) + t * G == stop_j) payload = S::value(w[t]);
                    }
                } else {
                    if (step == 0) step = probe_step<S::key_bytes, B>(a.probe, key);
                    idx = probe_next(idx, step, a.probe.capacity);
                    if (idx == init) done = true;
                }
            }
        }
        uint32_t const src = tile_shift + (stop_j >= 0 ? uint32_t(stop_j % G) : 0u);
        uint64_t const pv = __shfl_sync(0xffffffffu, (unsigned long long)payload, src);
        if (r == 0 && i < n) {
            if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = hit;
            else Io<S>::store_payload(out, i, hit ? pv : empty_payload<S>(a));
        }
    }
}

// ----------------------------------------------------------------------------
// Staged lookups: the key stream is brought into shared memory by bulk (TMA)
// copies, double-buffered, one 1024-key chunk per stage, so no lane waits on a
// key load before it can probe.  G lanes cooperate on a bucket window (one
// 16-byte slot per lane and round); each tile keeps Q windows in flight; the
// probe start index is hashed once per key (lane q of the tile) and shuffled.
// Keys of a pass are interleaved across tiles, so the tiles' first lanes
// store consecutive outputs.
// ----------------------------------------------------------------------------

constexpr uint32_t kStageKeys = 1024;

struct TileResult {
    uint64_t payload;
    bool hit;
    bool done;
};

// Resolves one loaded window of a tile (the whole warp calls it; tiles with
// `skip` set only take part in the ballots).  When the window ends the scan,
// the result has done set, the hit flag, and -- on every lane of the tile --
// the payload of the hit slot, handed over by the lane that loaded it.
template <class S, int B, int G, int ROUNDS>
__device__ __forceinline__ void tile_resolve(OaArgs const& a, typename S::Raw const (&w)[ROUNDS], uint64_t key,
                                             uint32_t r, uint32_t lane0, bool skip, TileResult& res)
{
    constexpr uint32_t MASK = (1u << G) - 1u;
    uint32_t stop_bits = 0, hit_bits = 0;
#pragma unroll
    for (int t = 0; t < ROUNDS; ++t) {
        bool const own = !skip && int(r) + t * G < B;
        uint64_t const k = own ? S::key(w[t]) : 0;
        bool const is_stop = own && (k == a.empty_key || S::key_eq(k, key));
        bool const is_hit = is_stop && k != a.empty_key;
        stop_bits |= ((__ballot_sync(0xffffffffu, is_stop) >> lane0) & MASK) << (t * G);
        hit_bits |= ((__ballot_sync(0xffffffffu, is_hit) >> lane0) & MASK) << (t * G);
    }
    int const stop_j = stop_bits ? __ffs(stop_bits) - 1 : -1;
    // the lane holding slot stop_j picks it by a compare per round: a select
    // keyed on stop_j / G becomes a dynamically indexed copy of w in local memory
    uint64_t mine = 0;
#pragma unroll
    for (int t = 0; t < ROUNDS; ++t)
        if (int(r) + t * G == stop_j) mine = S::value(w[t]);
    uint64_t const got = __shfl_sync(0xffffffffu, (unsigned long long)mine, lane0 + (stop_j >= 0 ? stop_j % G : 0));
    if (!skip && stop_j >= 0) {
        res.done = true;
        res.hit = (hit_bits >> stop_j) & 1u;
        res.payload = got;
    }
}

// Split scan of a first window (the SEG variant).  DRAM reads for random
// lookups arrive as whole fill units (64 bytes under ld_ro's hint), and an
// 80-byte bucket spans two or three of them; the split variant reads the part
// in the first unit, and the rest only for windows the first part did not
// settle.
//
// Slots [lo, hi) of a window, lane r holding slots lo + r + t*G (t < ROUNDS):
// loads them and finds the first one that ends the scan, as tile_resolve does
// for a whole window.
template <class S, int B, int G, int ROUNDS>
__device__ __forceinline__ void load_range(typename S::Raw const* slots, uint32_t idx, int lo, int hi, uint32_t r,
                                           bool skip, typename S::Raw (&w)[ROUNDS])
{
#pragma unroll
    for (int t = 0; t < ROUNDS; ++t)
        if (!skip && lo + int(r) + t * G < hi) w[t] = ld_ro(slots + idx + lo + r + t * G);
}

template <class S, int B, int G, int ROUNDS>
__device__ __forceinline__ void resolve_range(OaArgs const& a, typename S::Raw const (&w)[ROUNDS], int lo, int hi,
                                              uint64_t key, uint32_t r, uint32_t lane0, bool skip, TileResult& res)
{
    constexpr uint32_t MASK = (1u << G) - 1u;
    uint32_t stop_bits = 0, hit_bits = 0;
#pragma unroll
    for (int t = 0; t < ROUNDS; ++t) {
        bool const own = !skip && lo + int(r) + t * G < hi;
        uint64_t const k = own ? S::key(w[t]) : 0;
        bool const is_stop = own && (k == a.empty_key || S::key_eq(k, key));
        bool const is_hit = is_stop && k != a.empty_key;
        stop_bits |= ((__ballot_sync(0xffffffffu, is_stop) >> lane0) & MASK) << (t * G);
        hit_bits |= ((__ballot_sync(0xffffffffu, is_hit) >> lane0) & MASK) << (t * G);
    }
    int const s = stop_bits ? __ffs(stop_bits) - 1 : -1;
    uint64_t mine = 0;
#pragma unroll
    for (int t = 0; t < ROUNDS; ++t)
        if (int(r) + t * G == s) mine = S::value(w[t]);
    uint64_t const got = __shfl_sync(0xffffffffu, (unsigned long long)mine, lane0 + (s >= 0 ? s % G : 0));
    if (!skip && s >= 0) {
        res.done = true;
        res.hit = (hit_bits >> s) & 1u;
        res.payload = got;
    }
}

// DRAM fill unit of the read-only loads: ld_ro asks for 64-byte L2 fills.
constexpr int kFillBytes = 64;

// Slots of the window starting at `idx` before the next fill-unit boundary.
template <class S, int B>
__device__ __forceinline__ int slots_to_line_end(uint32_t idx)
{
    constexpr int per = kFillBytes / S::bytes;
    int const n1 = per - int(idx % per);
    return n1 < B ? n1 : B;
}

// Further windows of keys whose first window neither held the key nor an
// empty slot (rare at load factor 0.5); the whole warp iterates until every
// tile is done.
template <class S, int B, int G, int ROUNDS>
__device__ __forceinline__ TileResult tile_continue(OaArgs a, typename S::Raw const* slots, uint64_t key, uint32_t init,
                                                 uint32_t r, uint32_t lane0, TileResult res)
{
    uint32_t idx = init, step = 0;
    while (__any_sync(0xffffffffu, !res.done)) {
        typename S::Raw w[ROUNDS];
        if (!res.done) {
            if (step == 0) step = probe_step<S::key_bytes, B>(a.probe, key);
            idx = probe_next(idx, step, a.probe.capacity);
            if (idx == init) {
                res.done = true;  // full cycle: not present
                res.hit = false;
            } else {
#pragma unroll
                for (int t = 0; t < ROUNDS; ++t)
                    if (int(r) + t * G < B) w[t] = ld_ro(slots + idx + r + t * G);
            }
        }
        tile_resolve<S, B, G, ROUNDS>(a, w, key, r, lane0, res.done, res);
    }
    return res;
}

template <class S, int B, int G, int Q, bool CONTAINS, bool SEG>
__global__ void __launch_bounds__(256) k_find_staged(__grid_constant__ const OaArgs a, void const* keys, void* out, uint32_t n, WaitCtl wc)
{
    static_assert(Q <= G && G <= 8 && (G & (G - 1)) == 0, "tile shape");
    using Raw = typename S::Raw;
    using Key = typename Io<S>::Key;
    constexpr int ROUNDS = (B + G - 1) / G;
    constexpr uint32_t TILES = 256 / G;             // tiles per block
    constexpr uint32_t PASS = TILES * Q;            // keys per pass
    static_assert(kStageKeys % PASS == 0, "stage must hold whole passes");
    __shared__ alignas(128) Key sk[2][kStageKeys];
    __shared__ alignas(8) uint64_t bar[2];
    __shared__ alignas(8) uint64_t never;  // no thread or copy ever arrives on it (timeout test hook)

    Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
    uint32_t const lane = threadIdx.x & 31, r = lane % G, tile_lane0 = lane & ~uint32_t(G - 1);
    uint32_t const tile = threadIdx.x / G;
    uint32_t const chunks = n / kStageKeys;
    constexpr uint32_t kChunkBytes = kStageKeys * sizeof(Key);

    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init(&never, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && blockIdx.x < chunks) {
        mbar_arrive_expect_tx(&bar[0], kChunkBytes);
        bulk_g2s(sk[0], static_cast<Key const*>(keys) + uint64_t(blockIdx.x) * kStageKeys, kChunkBytes, &bar[0]);
    }
    uint32_t it = 0;
    bool failed = false;
    for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x, ++it) {
        uint32_t const b = it & 1;
        uint32_t const cn = c + gridDim.x;
        if (threadIdx.x == 0 && cn < chunks) {
            fence_proxy_async();  // the other buffer's generic reads (previous chunk) precede this copy
            mbar_arrive_expect_tx(&bar[b ^ 1], kChunkBytes);
            bulk_g2s(sk[b ^ 1], static_cast<Key const*>(keys) + uint64_t(cn) * kStageKeys, kChunkBytes, &bar[b ^ 1]);
        }
        // the whole block agrees on the outcome, so every lane leaves together
        bool const ok = wc.probe_timeout ? mbar_wait_bounded(&never, 0, wc.ns)
                                         : mbar_wait_bounded(&bar[b], (it >> 1) & 1, wc.ns);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        Key const* ks = sk[b];
        uint32_t const base = c * kStageKeys;
        for (uint32_t p = 0; p < kStageKeys; p += PASS) {
            // key q of this tile sits at p + q * TILES + tile
            uint64_t key[Q];
            uint32_t idx[Q], init[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) key[q] = ks[p + q * TILES + tile];
            uint32_t my_init = 0;
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (int(r) == q) my_init = probe_init<S::key_bytes, B>(a.probe, key[q]);
#pragma unroll
            for (int q = 0; q < Q; ++q) idx[q] = init[q] = __shfl_sync(0xffffffffu, my_init, tile_lane0 + q);
            if constexpr (SEG) {
                // phase 1: every key's first window up to its L2 line end, all in flight together
                Raw w[Q][ROUNDS];
                int hi1[Q];
                TileResult res[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    hi1[q] = slots_to_line_end<S, B>(idx[q]);
                    load_range<S, B, G, ROUNDS>(slots, idx[q], 0, hi1[q], r, false, w[q]);
                }
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    res[q] = TileResult{0, false, false};
                    resolve_range<S, B, G, ROUNDS>(a, w[q], 0, hi1[q], key[q], r, tile_lane0, false, res[q]);
                }
                // phase 2: the part in the next line, only for windows the first part did not settle
#pragma unroll
                for (int q = 0; q < Q; ++q)
                    load_range<S, B, G, ROUNDS>(slots, idx[q], hi1[q], B, r, res[q].done, w[q]);
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    if (__any_sync(0xffffffffu, !res[q].done && hi1[q] < B))
                        resolve_range<S, B, G, ROUNDS>(a, w[q], hi1[q], B, key[q], r, tile_lane0,
                                                       res[q].done || hi1[q] >= B, res[q]);
                    if (__any_sync(0xffffffffu, !res[q].done))  // rare: further windows
                        res[q] = tile_continue<S, B, G, ROUNDS>(a, slots, key[q], init[q], r, tile_lane0, res[q]);
                    if (r == 0) {
                        uint32_t const i = base + p + q * TILES + tile;
                        if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = res[q].hit;
                        else Io<S>::store_payload(out, i, res[q].hit ? res[q].payload : empty_payload<S>(a));
                    }
                }
                continue;
            }
            // all Q first windows in flight before any is resolved
            Raw w[Q][ROUNDS];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int t = 0; t < ROUNDS; ++t)
                    if (int(r) + t * G < B) w[q][t] = ld_ro(slots + idx[q] + r + t * G);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                TileResult res{0, false, false};
                tile_resolve<S, B, G, ROUNDS>(a, w[q], key[q], r, tile_lane0, false, res);
                if (__any_sync(0xffffffffu, !res.done))  // rare: some tile needs further windows
                    res = tile_continue<S, B, G, ROUNDS>(a, slots, key[q], init[q], r, tile_lane0, res);
                if (r == 0) {
                    uint32_t const i = base + p + q * TILES + tile;
                    if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = res.hit;
                    else Io<S>::store_payload(out, i, res.hit ? res.payload : empty_payload<S>(a));
                }
            }
        }
        __syncthreads();  // every lane is done with sk[b] before it is refilled
    }
    if (failed) {
        if (threadIdx.x == 0) {
            atomicExch(wc.status, kStatusTimeout);
            // let the copies still in flight land before the block exits (bounded again)
            uint32_t const c = blockIdx.x + it * gridDim.x;
            mbar_wait_bounded(&bar[it & 1], (it >> 1) & 1, 1000000000ull);
            if (c + gridDim.x < chunks) mbar_wait_bounded(&bar[(it + 1) & 1], ((it + 1) >> 1) & 1, 1000000000ull);
        }
        return;
    }
    // the ragged tail (< one stage) goes through direct loads, block 0 only
    if (blockIdx.x == 0 && chunks * kStageKeys < n) {
        for (uint32_t i0 = chunks * kStageKeys; i0 < n; i0 += TILES) {
            uint32_t const i = i0 + tile;
            bool const live = i < n;
            uint64_t const key = live ? Io<S>::load_key(keys, i) : 0;
            uint32_t const init0 = live ? probe_init<S::key_bytes, B>(a.probe, key) : 0;
            Raw w[ROUNDS];
            if (live) {
#pragma unroll
                for (int t = 0; t < ROUNDS; ++t)
                    if (int(r) + t * G < B) w[t] = ld_ro(slots + init0 + r + t * G);
            }
            TileResult res{0, false, !live};
            tile_resolve<S, B, G, ROUNDS>(a, w, key, r, tile_lane0, !live, res);
            if (__any_sync(0xffffffffu, !res.done))
                res = tile_continue<S, B, G, ROUNDS>(a, slots, key, init0, r, tile_lane0, res);
            if (r == 0 && live) {
                if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = res.hit;
                else Io<S>::store_payload(out, i, res.hit ? res.payload : empty_payload<S>(a));
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Warp-staged lookups: like k_find_staged, but every warp stages its own
// 256-key chunks (double-buffered bulk copies, one mbarrier per buffer), so
// warps never wait for each other -- no block barrier, no straggler stalls
// when one warp's keys need further windows.
// ----------------------------------------------------------------------------

constexpr uint32_t kWarpStageKeys = 256;

template <class S, int B, int G, int Q, bool CONTAINS>
__global__ void __launch_bounds__(256, 4) k_find_wstaged(__grid_constant__ const OaArgs a, void const* keys, void* out, uint32_t n, WaitCtl wc)
{
    static_assert(Q <= G && G <= 8 && (G & (G - 1)) == 0, "tile shape");
    using Raw = typename S::Raw;
    using Key = typename Io<S>::Key;
    constexpr int ROUNDS = (B + G - 1) / G;
    constexpr uint32_t TILES = 32 / G;   // tiles per warp
    constexpr uint32_t PASS = TILES * Q;  // keys per warp pass
    static_assert(kWarpStageKeys % PASS == 0, "stage must hold whole passes");
    constexpr uint32_t kChunkBytes = kWarpStageKeys * sizeof(Key);
    __shared__ alignas(128) Key sk[8][2][kWarpStageKeys];
    __shared__ alignas(8) uint64_t bar[8][2];
    __shared__ alignas(8) uint64_t never[8];

    Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
    uint32_t const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t const r = lane % G, tile_lane0 = lane & ~uint32_t(G - 1), tile = lane / G;
    uint32_t const gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t const nwarps = (gridDim.x * blockDim.x) >> 5;
    uint32_t const chunks = n / kWarpStageKeys;
    Key const* kin = static_cast<Key const*>(keys);

    if (lane == 0) {
        mbar_init(&bar[warp][0], 1);
        mbar_init(&bar[warp][1], 1);
        mbar_init(&never[warp], 1);
        fence_mbar_init();
        if (gwarp < chunks) {
            mbar_arrive_expect_tx(&bar[warp][0], kChunkBytes);
            bulk_g2s(sk[warp][0], kin + uint64_t(gwarp) * kWarpStageKeys, kChunkBytes, &bar[warp][0]);
        }
    }
    __syncwarp();
    uint32_t it = 0;
    bool failed = false;
    for (uint32_t c = gwarp; c < chunks; c += nwarps, ++it) {
        uint32_t const b = it & 1;
        uint32_t const cn = c + nwarps;
        if (lane == 0 && cn < chunks) {
            fence_proxy_async();  // the warp's reads of this buffer (previous chunk) precede the copy
            mbar_arrive_expect_tx(&bar[warp][b ^ 1], kChunkBytes);
            bulk_g2s(sk[warp][b ^ 1], kin + uint64_t(cn) * kWarpStageKeys, kChunkBytes, &bar[warp][b ^ 1]);
        }
        bool const ok = wc.probe_timeout ? mbar_wait_bounded(&never[warp], 0, wc.ns)
                                         : mbar_wait_bounded(&bar[warp][b], (it >> 1) & 1, wc.ns);
        if (__any_sync(0xffffffffu, !ok)) {
            failed = true;
            break;
        }
        Key const* ks = sk[warp][b];
        uint32_t const base = c * kWarpStageKeys;
        for (uint32_t p = 0; p < kWarpStageKeys; p += PASS) {
            uint64_t key[Q];
            uint32_t idx[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) key[q] = ks[p + q * TILES + tile];
            uint32_t my_init = 0;
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (int(r) == q) my_init = probe_init<S::key_bytes, B>(a.probe, key[q]);
#pragma unroll
            for (int q = 0; q < Q; ++q) idx[q] = __shfl_sync(0xffffffffu, my_init, tile_lane0 + q);
            Raw w[Q][ROUNDS];
#pragma unroll
            for (int q = 0; q < Q; ++q) load_range<S, B, G, ROUNDS>(slots, idx[q], 0, B, r, false, w[q]);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                TileResult res{0, false, false};
                resolve_range<S, B, G, ROUNDS>(a, w[q], 0, B, key[q], r, tile_lane0, false, res);
                if (__any_sync(0xffffffffu, !res.done))  // rare: further windows
                    res = tile_continue<S, B, G, ROUNDS>(a, slots, key[q], idx[q], r, tile_lane0, res);
                if (r == 0) {
                    uint32_t const i = base + p + q * TILES + tile;
                    if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = res.hit;
                    else Io<S>::store_payload(out, i, res.hit ? res.payload : empty_payload<S>(a));
                }
            }
        }
        __syncwarp();  // every lane is done with this buffer before it is refilled
    }
    if (failed) {
        if (lane == 0) {
            atomicExch(wc.status, kStatusTimeout);
            // let this warp's copies still in flight land before the block can exit (bounded again)
            uint32_t const c = gwarp + it * nwarps;
            mbar_wait_bounded(&bar[warp][it & 1], (it >> 1) & 1, 1000000000ull);
            if (c + nwarps < chunks) mbar_wait_bounded(&bar[warp][(it + 1) & 1], ((it + 1) >> 1) & 1, 1000000000ull);
        }
        return;
    }
    // the ragged tail (< one warp stage) goes to one warp, keys read directly
    if (chunks * kWarpStageKeys < n && gwarp == chunks % nwarps) {
        for (uint32_t i0 = chunks * kWarpStageKeys; i0 < n; i0 += TILES) {
            uint32_t const i = i0 + tile;
            bool const live = i < n;
            uint64_t const key = live ? Io<S>::load_key(keys, i) : 0;
            uint32_t const init0 = live ? probe_init<S::key_bytes, B>(a.probe, key) : 0;
            Raw w[ROUNDS];
            load_range<S, B, G, ROUNDS>(slots, init0, 0, B, r, !live, w);
            TileResult res{0, false, !live};
            resolve_range<S, B, G, ROUNDS>(a, w, 0, B, key, r, tile_lane0, !live, res);
            if (__any_sync(0xffffffffu, !res.done))
                res = tile_continue<S, B, G, ROUNDS>(a, slots, key, init0, r, tile_lane0, res);
            if (r == 0 && live) {
                if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = res.hit;
                else Io<S>::store_payload(out, i, res.hit ? res.payload : empty_payload<S>(a));
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Deferred-continuation lookups: keys staged per warp as in k_find_wstaged, but
// a key whose first window holds neither the key nor an empty slot is queued in
// the warp's shared-memory ring instead of being followed at once, so a pass
// costs one dependent window load however many of its keys probe on.  Once a
// whole pass of keys is queued the warp follows them together, one window each,
// and queues again the few that need yet another.  A tile resolves a window
// without ballots: each lane finds the first slot among its own that ends the
// scan, a min over the tile's lanes gives the window's first, and the lane
// holding that slot writes the result.
// ----------------------------------------------------------------------------

constexpr uint32_t kDeferRing = 64;  // queued keys per warp (a power of two)
constexpr int kNoStop = 255;

// First slot of a window (lane r holds slots r + t*G) that ends the scan of
// `key`, agreed by the tile's G lanes, or kNoStop.  `own` is the lane's own
// first such slot (kNoStop if none) and `mine` that slot's contents.  Lanes of
// tiles with `skip` set only take part in the shuffles.
template <class S, int B, int G, int ROUNDS>
__device__ __forceinline__ int tile_first_stop(typename S::Raw const (&w)[ROUNDS], bool skip, uint64_t key,
                                               uint64_t empty_key, uint32_t r, int& own, typename S::Raw& mine)
{
    own = kNoStop;
#pragma unroll
    for (int t = ROUNDS - 1; t >= 0; --t) {
        if (!skip && int(r) + t * G < B) {
            uint64_t const k = S::key(w[t]);
            if (k == empty_key || S::key_eq(k, key)) {
                own = int(r) + t * G;
                mine = w[t];
            }
        }
    }
    int s = own;
#pragma unroll
    for (int o = 1; o < G; o <<= 1) s = min(s, __shfl_xor_sync(0xffffffffu, s, o));
    return s;
}

// Resident blocks per SM the deferred lookup is compiled for (register cap).
#ifndef B2CO_WDEFER_MINB
#define B2CO_WDEFER_MINB(Q) ((Q) == 1 ? 4 : 3)
#endif

template <class S, int B, int G, int Q, bool CONTAINS>
__global__ void __launch_bounds__(256, B2CO_WDEFER_MINB(Q)) k_find_wdefer(__grid_constant__ const OaArgs a, void const* keys, void* out,
                                                        uint32_t n, WaitCtl wc)
{
    static_assert(Q <= G && G <= 8 && (G & (G - 1)) == 0, "tile shape");
    using Raw = typename S::Raw;
    using Key = typename Io<S>::Key;
    constexpr int ROUNDS = (B + G - 1) / G;
    constexpr uint32_t TILES = 32 / G;   // tiles per warp
    constexpr uint32_t PASS = TILES * Q;  // keys per warp pass
    static_assert(kWarpStageKeys % PASS == 0, "stage must hold whole passes");
    static_assert(2 * PASS <= kDeferRing, "the ring must hold a pass on top of a partial one");
    constexpr uint32_t RING = kDeferRing - 1;
    constexpr uint32_t kChunkBytes = kWarpStageKeys * sizeof(Key);
    __shared__ alignas(128) Key sk[8][2][kWarpStageKeys];
    __shared__ alignas(8) uint64_t bar[8][2];
    __shared__ alignas(8) uint64_t never[8];
    // the warp's queue of keys still probing: key, first window, last window read, output index
    __shared__ uint64_t qkey[8][kDeferRing];
    __shared__ uint32_t qinit[8][kDeferRing], qidx[8][kDeferRing], qpos[8][kDeferRing];

    Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
    uint32_t const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t const r = lane % G, tile_lane0 = lane & ~uint32_t(G - 1), tile = lane / G;
    uint32_t const gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t const nwarps = (gridDim.x * blockDim.x) >> 5;
    uint32_t const chunks = n / kWarpStageKeys;
    Key const* kin = static_cast<Key const*>(keys);
    uint32_t head = 0, count = 0;  // queue state, the same on every lane

    auto settle = [&](uint32_t pos, Raw const& slot) {  // result from the slot that ended the scan
        bool const hit = S::key(slot) != a.empty_key;
        if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[pos] = hit;
        else Io<S>::store_payload(out, pos, hit ? S::value(slot) : empty_payload<S>(a));
    };
    auto settle_miss = [&](uint32_t pos) {
        if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[pos] = 0;
        else Io<S>::store_payload(out, pos, empty_payload<S>(a));
    };
    // Lane 0 of each tile whose window ended no scan queues its key.
    auto enqueue = [&](bool unsettled, uint64_t key, uint32_t init, uint32_t idx, uint32_t pos) {
        uint32_t const m = __ballot_sync(0xffffffffu, unsettled);
        if (unsettled) {
            uint32_t const e = (head + count + __popc(m & ((1u << lane) - 1u))) & RING;
            qkey[warp][e] = key;
            qinit[warp][e] = init;
            qidx[warp][e] = idx;
            qpos[warp][e] = pos;
        }
        count += __popc(m);
    };
    // Takes up to one pass of queued keys and reads the next window of each.
    auto follow = [&]() {
        __syncwarp();  // the queue writes precede these reads
        uint32_t const take = count < PASS ? count : PASS;
        uint64_t key[Q];
        uint32_t init[Q], idx[Q], pos[Q];
        bool live[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint32_t const j = q * TILES + tile;
            live[q] = j < take;
            uint32_t const e = (head + (live[q] ? j : 0u)) & RING;
            key[q] = qkey[warp][e];
            init[q] = qinit[warp][e];
            idx[q] = qidx[warp][e];
            pos[q] = qpos[warp][e];
        }
        __syncwarp();  // every read of the taken entries precedes their reuse
        head = (head + take) & RING;
        count -= take;
        uint32_t my_step = 0;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (int(r) == q && live[q]) my_step = probe_step<S::key_bytes, B>(a.probe, key[q]);
        Raw w[Q][ROUNDS];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint32_t const step = __shfl_sync(0xffffffffu, my_step, tile_lane0 + q);
            if (live[q]) {
                idx[q] = probe_next(idx[q], step, a.probe.capacity);
                if (idx[q] == init[q]) {  // full cycle: not present
                    if (r == 0) settle_miss(pos[q]);
                    live[q] = false;
                }
            }
            load_range<S, B, G, ROUNDS>(slots, idx[q], 0, B, r, !live[q], w[q]);
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int own;
            Raw mine{};
            int const s = tile_first_stop<S, B, G, ROUNDS>(w[q], !live[q], key[q], a.empty_key, r, own, mine);
            if (live[q] && s != kNoStop && own == s) settle(pos[q], mine);
            enqueue(live[q] && s == kNoStop && r == 0, key[q], init[q], idx[q], pos[q]);
        }
    };

    if (lane == 0) {
        mbar_init(&bar[warp][0], 1);
        mbar_init(&bar[warp][1], 1);
        mbar_init(&never[warp], 1);
        fence_mbar_init();
        if (gwarp < chunks) {
            mbar_arrive_expect_tx(&bar[warp][0], kChunkBytes);
            bulk_g2s(sk[warp][0], kin + uint64_t(gwarp) * kWarpStageKeys, kChunkBytes, &bar[warp][0]);
        }
    }
    __syncwarp();
    uint32_t it = 0;
    bool failed = false;
    for (uint32_t c = gwarp; c < chunks; c += nwarps, ++it) {
        uint32_t const b = it & 1;
        uint32_t const cn = c + nwarps;
        if (lane == 0 && cn < chunks) {
            fence_proxy_async();  // the warp's reads of this buffer (previous chunk) precede the copy
            mbar_arrive_expect_tx(&bar[warp][b ^ 1], kChunkBytes);
            bulk_g2s(sk[warp][b ^ 1], kin + uint64_t(cn) * kWarpStageKeys, kChunkBytes, &bar[warp][b ^ 1]);
        }
        bool const ok = wc.probe_timeout ? mbar_wait_bounded(&never[warp], 0, wc.ns)
                                         : mbar_wait_bounded(&bar[warp][b], (it >> 1) & 1, wc.ns);
        if (__any_sync(0xffffffffu, !ok)) {
            failed = true;
            break;
        }
        Key const* ks = sk[warp][b];
        uint32_t const base = c * kWarpStageKeys;
        for (uint32_t p = 0; p < kWarpStageKeys; p += PASS) {
            uint64_t key[Q];
            uint32_t idx[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) key[q] = ks[p + q * TILES + tile];
            uint32_t my_init = 0;
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (int(r) == q) my_init = probe_init<S::key_bytes, B>(a.probe, key[q]);
#pragma unroll
            for (int q = 0; q < Q; ++q) idx[q] = __shfl_sync(0xffffffffu, my_init, tile_lane0 + q);
            Raw w[Q][ROUNDS];
#pragma unroll
            for (int q = 0; q < Q; ++q) load_range<S, B, G, ROUNDS>(slots, idx[q], 0, B, r, false, w[q]);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                int own;
                Raw mine{};
                int const s = tile_first_stop<S, B, G, ROUNDS>(w[q], false, key[q], a.empty_key, r, own, mine);
                uint32_t const i = base + p + q * TILES + tile;
                if (s != kNoStop && own == s) settle(i, mine);
                enqueue(s == kNoStop && r == 0, key[q], idx[q], idx[q], i);
            }
            while (count >= PASS) follow();
        }
        __syncwarp();  // every lane is done with this buffer before it is refilled
    }
    if (failed) {
        if (lane == 0) {
            atomicExch(wc.status, kStatusTimeout);
            // let this warp's copies still in flight land before the block can exit (bounded again)
            uint32_t const c = gwarp + it * nwarps;
            mbar_wait_bounded(&bar[warp][it & 1], (it >> 1) & 1, 1000000000ull);
            if (c + nwarps < chunks) mbar_wait_bounded(&bar[warp][(it + 1) & 1], ((it + 1) >> 1) & 1, 1000000000ull);
        }
        return;
    }
    while (count > 0) follow();  // each round moves every queued key on by a window or settles it
    // the ragged tail (< one warp stage) goes to one warp, keys read directly
    if (chunks * kWarpStageKeys < n && gwarp == chunks % nwarps) {
        for (uint32_t i0 = chunks * kWarpStageKeys; i0 < n; i0 += TILES) {
            uint32_t const i = i0 + tile;
            bool const live = i < n;
            uint64_t const key = live ? Io<S>::load_key(keys, i) : 0;
            uint32_t const init0 = live ? probe_init<S::key_bytes, B>(a.probe, key) : 0;
            Raw w[ROUNDS];
            load_range<S, B, G, ROUNDS>(slots, init0, 0, B, r, !live, w);
            TileResult res{0, false, !live};
            resolve_range<S, B, G, ROUNDS>(a, w, 0, B, key, r, tile_lane0, !live, res);
            if (__any_sync(0xffffffffu, !res.done))
                res = tile_continue<S, B, G, ROUNDS>(a, slots, key, init0, r, tile_lane0, res);
            if (r == 0 && live) {
                if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = res.hit;
                else Io<S>::store_payload(out, i, res.hit ? res.payload : empty_payload<S>(a));
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Bulk-window lookups (16-byte slots): every lane fetches its key's whole first
// bucket window (B x 16 bytes, 16-byte aligned) with ONE bulk copy (TMA,
// untiled) into shared memory.  Copies are tracked by the SM's bulk-copy
// engine instead of the load/store unit, so a block keeps a whole stage of
// 1024 windows in flight.  The 32 lanes of a warp arrive on one mbarrier per
// batch; a lane resolves its own window from shared memory, and the rare key
// that needs further windows continues with direct loads.  Keys are staged
// by the same double-buffered bulk copies as k_find_staged.
// ----------------------------------------------------------------------------

constexpr int kBulkBatches = kStageKeys / 256;  // batches of 32 windows per warp per stage

template <class S, int B>
__host__ __device__ constexpr uint32_t bulk_window_smem()
{
    return 8u * kBulkBatches * 32u * uint32_t(B) * 16u;  // 8 warps x batches x 32 lanes x window
}

template <class S, int B, bool CONTAINS>
__global__ void __launch_bounds__(256) k_find_bulk(__grid_constant__ const OaArgs a, void const* keys, void* out, uint32_t n, WaitCtl wc)
{
    static_assert(S::bytes == 16, "bulk windows need 16-byte slots (16-byte aligned windows)");
    using Raw = typename S::Raw;
    using Key = typename Io<S>::Key;
    constexpr uint32_t WIN = uint32_t(B) * 16u;
    __shared__ alignas(128) Key sk[2][kStageKeys];
    __shared__ alignas(8) uint64_t kbar[2];
    __shared__ alignas(8) uint64_t wbar[8][kBulkBatches];
    __shared__ alignas(8) uint64_t never;
    extern __shared__ __align__(128) unsigned char wins[];  // [warp][batch][lane][WIN]

    Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
    uint32_t const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t const chunks = n / kStageKeys;
    constexpr uint32_t kChunkBytes = kStageKeys * sizeof(Key);

    if (threadIdx.x == 0) {
        mbar_init(&kbar[0], 1);
        mbar_init(&kbar[1], 1);
        mbar_init(&never, 1);
        for (int w = 0; w < 8; ++w)
            for (int j = 0; j < kBulkBatches; ++j) mbar_init(&wbar[w][j], 32);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && blockIdx.x < chunks) {
        mbar_arrive_expect_tx(&kbar[0], kChunkBytes);
        bulk_g2s(sk[0], static_cast<Key const*>(keys) + uint64_t(blockIdx.x) * kStageKeys, kChunkBytes, &kbar[0]);
    }
    uint32_t it = 0;
    bool failed = false, issued = false;
    for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x, ++it) {
        uint32_t const b = it & 1;
        uint32_t const cn = c + gridDim.x;
        issued = false;
        if (threadIdx.x == 0 && cn < chunks) {
            fence_proxy_async();
            mbar_arrive_expect_tx(&kbar[b ^ 1], kChunkBytes);
            bulk_g2s(sk[b ^ 1], static_cast<Key const*>(keys) + uint64_t(cn) * kStageKeys, kChunkBytes, &kbar[b ^ 1]);
        }
        bool ok = wc.probe_timeout ? mbar_wait_bounded(&never, 0, wc.ns)
                                   : mbar_wait_bounded(&kbar[b], (it >> 1) & 1, wc.ns);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        issued = true;
        Key const* ks = sk[b];
        uint32_t const base = c * kStageKeys;
        // issue every window copy of this warp's share of the stage
        uint64_t key[kBulkBatches];
        uint32_t init[kBulkBatches];
        unsigned char* my_win = wins + (size_t(warp) * kBulkBatches * 32 + lane) * WIN;
        fence_proxy_async();  // the previous stage's reads of the windows precede the new copies
#pragma unroll
        for (int j = 0; j < kBulkBatches; ++j) {
            uint32_t const pos = (warp * kBulkBatches + j) * 32 + lane;
            key[j] = ks[pos];
            init[j] = probe_init<S::key_bytes, B>(a.probe, key[j]);
            mbar_arrive_expect_tx(&wbar[warp][j], WIN);
            bulk_g2s(my_win + size_t(j) * 32 * WIN, slots + init[j], WIN, &wbar[warp][j]);
        }
        // resolve batch by batch as the windows land
#pragma unroll
        for (int j = 0; j < kBulkBatches; ++j) {
            ok = mbar_wait_bounded(&wbar[warp][j], it & 1, wc.ns);
            uint32_t const pos = (warp * kBulkBatches + j) * 32 + lane;
            uint64_t payload = empty_payload<S>(a);
            bool hit = false;
            if (ok) {
                Raw const* w = reinterpret_cast<Raw const*>(my_win + size_t(j) * 32 * WIN);
                int stop = -1;
#pragma unroll
                for (int s = B - 1; s >= 0; --s) {
                    uint64_t k = S::key(w[s]);
                    if (k == a.empty_key || S::key_eq(k, key[j])) stop = s;
                }
                if (stop >= 0) {
                    hit = S::key(w[stop]) != a.empty_key;
                    if (hit) payload = S::value(w[stop]);
                } else {
                    hit = find_rest<S, B>(a, key[j], init[j], payload);
                }
            } else {
                failed = true;
            }
            if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[base + pos] = hit;
            else Io<S>::store_payload(out, base + pos, hit ? payload : empty_payload<S>(a));
        }
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
    }
    if (failed) {
        atomicExch(wc.status, kStatusTimeout);
        // let this lane's and this block's copies land before the block exits (bounded again)
        if (issued) {
#pragma unroll
            for (int j = 0; j < kBulkBatches; ++j) mbar_wait_bounded(&wbar[warp][j], it & 1, 1000000000ull);
        }
        if (threadIdx.x == 0) {
            mbar_wait_bounded(&kbar[it & 1], (it >> 1) & 1, 1000000000ull);
            if (blockIdx.x + (it + 1) * gridDim.x < chunks)
                mbar_wait_bounded(&kbar[(it + 1) & 1], ((it + 1) >> 1) & 1, 1000000000ull);
        }
        return;
    }
    // ragged tail: block 0, one lane per key, direct loads
    if (blockIdx.x == 0) {
        for (uint32_t i = chunks * kStageKeys + threadIdx.x; i < n; i += blockDim.x) {
            uint64_t const key = Io<S>::load_key(keys, i);
            uint32_t const init0 = probe_init<S::key_bytes, B>(a.probe, key);
            Raw w[B];
            load_window<S, B>(slots, init0, w);
            Raw stop;
            uint64_t payload = empty_payload<S>(a);
            bool hit;
            if (scan_window<S, B>(w, key, a.empty_key, stop)) {
                hit = S::key(stop) != a.empty_key;
                if (hit) payload = S::value(stop);
            } else {
                hit = find_rest<S, B>(a, key, init0, payload);
            }
            if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = hit;
            else Io<S>::store_payload(out, i, hit ? payload : empty_payload<S>(a));
        }
    }
}

// ----------------------------------------------------------------------------
// Erase (open_addressing_ref_impl.h:340-379) and Count (kernels.h:427-467)
// ----------------------------------------------------------------------------

template <class S, int B>
__global__ void __launch_bounds__(256) k_erase(__grid_constant__ const OaArgs a, void const* keys, uint32_t n, unsigned long long* counters)
{
    using Raw = typename S::Raw;
    Raw* slots = reinterpret_cast<Raw*>(a.slots);
    bool const tomb = a.erased_key != a.empty_key;
    uint64_t const target_key = tomb ? a.erased_key : a.empty_key;
    uint32_t failed = 0;
    uint32_t const stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        uint32_t i = base + (threadIdx.x & 31);
        if (i >= n) continue;
        uint64_t key = Io<S>::load_key(keys, i);
        uint32_t const init = probe_init<S::key_bytes, B>(a.probe, key);
        uint32_t idx = init, step = 0;
        bool done = false, ok = false;
        while (!done) {
#pragma unroll
            for (int j = 0; j < B; ++j) {
                if (done) break;
                Raw* sp = slots + idx + j;
                Raw cur = ld_rw(sp);
                uint64_t k = S::key(cur);
                if (k == a.empty_key) {
                    // only a configured tombstone lets an empty slot end the search
                    if (tomb) done = true;
                    continue;
                }
                if (S::key_eq(k, key)) {
                    Raw desired;
                    if constexpr (S::bytes == 16) desired = insert_desired<S>(cur, target_key, a.empty_value);
                    else desired = S::make(target_key, a.empty_value);
                    Raw old = cas_slot(sp, cur, desired);
                    if (raw_eq(old, cur)) {
                        ok = true;
                        done = true;
                    } else if (S::key(old) == target_key) {
                        done = true;  // another thread erased it first
                    }
                }
            }
            if (done) break;
            if (step == 0) step = probe_step<S::key_bytes, B>(a.probe, key);
            idx = probe_next(idx, step, a.probe.capacity);
            if (idx == init) break;
        }
        failed += !ok;
    }
    if (counters) warp_add_counter(counters, failed);
}

template <class S, int B>
__global__ void __launch_bounds__(256) k_count(__grid_constant__ const OaArgs a, void const* keys, uint32_t n, unsigned long long* counter)
{
    using Raw = typename S::Raw;
    Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
    uint32_t c = 0;
    uint32_t const stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        uint32_t i = base + (threadIdx.x & 31);
        if (i >= n) continue;
        uint64_t key = Io<S>::load_key(keys, i);
        uint32_t init = probe_init<S::key_bytes, B>(a.probe, key);
        Raw w[B];
        load_window<S, B>(slots, init, w);
        Raw stop;
        uint64_t payload;
        if (scan_window<S, B>(w, key, a.empty_key, stop)) c += S::key(stop) != a.empty_key;
        else c += find_rest<S, B>(a, key, init, payload);
    }
    warp_add_counter(counter, c);
}

// ----------------------------------------------------------------------------
// Clear: every slot becomes the empty pair, padding bytes zero
// (bucket_storage.inl:52-64, open_addressing_impl.h:478-499)
// ----------------------------------------------------------------------------

template <class S>
__global__ void __launch_bounds__(256) k_clear(void* slots, uint32_t capacity, uint64_t empty_key, uint64_t empty_value)
{
    using Raw = typename S::Raw;
    Raw const e = S::make(empty_key, empty_value);
    Raw* s = reinterpret_cast<Raw*>(slots);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < capacity; i += gridDim.x * blockDim.x) s[i] = e;
}

}  // namespace b2co
