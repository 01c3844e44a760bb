// oa_inst.cuh -- launchers of the open-addressing kernels for one slot layout.
// Each oa_slot_*.cu instantiates this for one layout so the six layouts
// compile in parallel.
#pragma once

#include "b2co_host.h"
#include "group_kernels.cuh"
#include "oa_insert.cuh"
#include "oa_kernels.cuh"

namespace b2co {

template <class S>
struct OaImpl {
    static constexpr uint32_t kBlock = 256;
    // The integer 4- and 8-byte layouts compile every lookup and write shape;
    // 2-byte and floating-point-key layouts compile the default shapes only
    // (another requested shape runs the default one).
    static constexpr bool kAllShapes = !S::float_key && S::key_bytes >= 4;

    template <class F>
    static int with_b(uint32_t b, F&& f)
    {
        switch (b) {
            case 1: return f(std::integral_constant<int, 1>{});
            case 2: return f(std::integral_constant<int, 2>{});
            case 4: return f(std::integral_constant<int, 4>{});
            case 5: return f(std::integral_constant<int, 5>{});
            case 8: return f(std::integral_constant<int, 8>{});
        }
        return fail(B2CO_EINVAL, "unsupported bucket size");
    }

    static int check_launch(char const* what)
    {
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? B2CO_OK : cuda_fail(e, what);
    }

    static int clear(OaArgs const& a, cudaStream_t s)
    {
        auto k = k_clear<S>;
        k<<<grid_for((void const*)k, kBlock, a.probe.capacity, kBlock * 4), kBlock, 0, s>>>(
            a.slots, a.probe.capacity, a.empty_key, a.empty_value);
        return check_launch("clear kernel");
    }

    // Whether the insert family runs one key per lane (the scan of
    // open_addressing_ref_impl.h:489-532 as written) instead of a tile per window.
    static bool per_key_writes(OaArgs const& a, int B) { return B == 1 || (a.write_shape >> 8) == 1; }

    // Cooperative-window write kernel (oa_insert.cuh) of the table's shape.
    template <int B, int MODE>
    static int launch_write(OaArgs const& a, void const* pairs, uint8_t const* stencil, uint32_t n, InsOut const& o,
                            cudaStream_t s)
    {
        uint32_t lanes = a.write_shape >> 8, items = a.write_shape & 0xffu;
        if (lanes == 0) lanes = 4, items = 1;  // default: 4 lanes per window, one key per lane group
        void (*k)(OaArgs, void const*, uint8_t const*, uint32_t, InsOut) = nullptr;
        if constexpr (kAllShapes && B == 5) {  // other shapes: the common bucket size only (build time)
            if (lanes == 2) k = items >= 2 ? k_insert_win<S, B, 2, 2, MODE> : k_insert_win<S, B, 2, 1, MODE>;
            else if (lanes == 8) k = items >= 4 ? k_insert_win<S, B, 8, 4, MODE> : k_insert_win<S, B, 8, 2, MODE>;
            else if (items == 2) k = k_insert_win<S, B, 4, 2, MODE>;
            else if (items >= 4) k = k_insert_win<S, B, 4, 4, MODE>;
        }
        if (!k) lanes = 4, items = 1, k = k_insert_win<S, B, 4, 1, MODE>;
        uint64_t const per_block = (kBlock / 32) * (32 / lanes) * items;
        k<<<grid_for((void const*)k, kBlock, n, per_block), kBlock, 0, s>>>(a, pairs, stencil, n, o);
        return check_launch("insert kernel");
    }

    static int insert(OaArgs const& a, uint32_t b, void const* pairs, uint8_t const* stencil, uint32_t n,
                      bool assign, unsigned long long* counters, cudaStream_t s)
    {
        return with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            if constexpr (B > 1) {
                if (!per_key_writes(a, B)) {
                    InsOut o{};
                    o.counters = counters;
                    return assign ? launch_write<B, kInsAssign>(a, pairs, stencil, n, o, s)
                                  : launch_write<B, kInsPlain>(a, pairs, stencil, n, o, s);
                }
            }
            auto k = assign ? k_insert<S, B, true> : k_insert<S, B, false>;
            k<<<grid_for((void const*)k, kBlock, n, kBlock), kBlock, 0, s>>>(a, pairs, stencil, n, counters);
            return check_launch("insert kernel");
        });
    }

    static int assign_if(OaArgs const& a, uint32_t b, void const* pairs, uint8_t const* stencil, uint32_t n,
                         cudaStream_t s)
    {
        return with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            auto k = k_assign_if<S, B>;
            k<<<grid_for((void const*)k, kBlock, n, kBlock), kBlock, 0, s>>>(a, pairs, stencil, n);
            return check_launch("assign kernel");
        });
    }

    static int iaf_race(OaArgs const& a, uint32_t b, void const* pairs, void* found, uint8_t* inserted, uint32_t n,
                        cudaStream_t s)
    {
        return with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            if constexpr (B > 1) {
                if (!per_key_writes(a, B)) {
                    InsOut o{};
                    o.found = found;
                    o.inserted = inserted;
                    return launch_write<B, kInsIafRace>(a, pairs, nullptr, n, o, s);
                }
            }
            auto k = k_iaf_race<S, B>;
            k<<<grid_for((void const*)k, kBlock, n, kBlock), kBlock, 0, s>>>(a, pairs, found, inserted, n);
            return check_launch("insert_and_find kernel");
        });
    }

    static int iaf_first(OaArgs const& a, uint32_t b, void const* pairs, void* found, uint8_t* inserted,
                         uint32_t n, uint32_t* pos, uint32_t* newbits, uint32_t* owner, cudaStream_t s)
    {
        return with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            // `newbits` holds two bitmaps of the table's slots: claimed in this
            // batch, then shared with later inputs of the batch (`dup`)
            uint32_t* dup = newbits + (uint64_t(a.probe.capacity) + 31) / 32;
            uint32_t const claim_bit = a.probe.capacity < kClaimBit ? kClaimBit : 0u;  // slot indices below 2^31 - 1
            bool placed = false;
            if constexpr (B > 1) {
                if (!per_key_writes(a, B)) {
                    InsOut o{};
                    o.pos = pos;
                    o.newbits = newbits;
                    o.owner = owner;
                    o.claim_bit = claim_bit;
                    if (int st = launch_write<B, kInsIafPlace>(a, pairs, nullptr, n, o, s)) return st;
                    placed = true;
                }
            }
            if (!placed) {
                auto k1 = k_iaf_place<S, B>;
                k1<<<grid_for((void const*)k1, kBlock, n, kBlock), kBlock, 0, s>>>(a, pairs, n, pos, newbits, owner,
                                                                                    claim_bit);
            }
            auto const grid = [&](void const* k) { return grid_for(k, kBlock, (uint64_t(n) + 3) / 4, kBlock); };
            k_iaf_min<S><<<grid((void const*)k_iaf_min<S>), kBlock, 0, s>>>(pos, newbits, dup, owner, n, claim_bit);
            if (claim_bit)
                k_iaf_claim<S><<<grid((void const*)k_iaf_claim<S>), kBlock, 0, s>>>(pos, dup, owner, n, claim_bit);
            auto k3 = k_iaf_final<S>;
            k3<<<grid((void const*)k3), kBlock, 0, s>>>(a, pairs, pos, newbits, dup, owner, found, inserted, n,
                                                        claim_bit);
            if (claim_bit) {
                // owner[] back to all-ones: a batch within 8x of the table's slots
                // clears the whole array (one sequential write) rather than
                // visiting its shared slots at random
                if (uint64_t(a.probe.capacity) <= 8ull * n) {
                    cudaError_t const e = cudaMemsetAsync(owner, 0xff, uint64_t(a.probe.capacity) * 4, s);
                    if (e != cudaSuccess) return cuda_fail(e, "insert_and_find (first wins) owner reset");
                } else {
                    k_iaf_restore<S><<<grid((void const*)k_iaf_restore<S>), kBlock, 0, s>>>(pos, dup, owner, n,
                                                                                             claim_bit);
                }
            }
            return check_launch("insert_and_find (first wins) kernels");
        });
    }

    template <int B, int G, bool C, bool SEG>
    static int find_staged(OaArgs const& a, uint32_t items, void const* keys, void* out, uint32_t n, WaitCtl wc,
                           cudaStream_t s)
    {
        void (*k)(OaArgs, void const*, void*, uint32_t, WaitCtl) = nullptr;
        if (items >= 4 && G >= 4) k = k_find_staged<S, B, G, (G >= 4 ? 4 : 1), C, SEG>;
        else if (items >= 2) k = k_find_staged<S, B, G, 2, C, SEG>;
        else k = k_find_staged<S, B, G, 1, C, SEG>;
        uint64_t chunks = n / kStageKeys;
        uint32_t grid = grid_for((void const*)k, kBlock, chunks ? chunks : 1, 1);
        k<<<grid, kBlock, 0, s>>>(a, keys, out, n, wc);
        return check_launch(C ? "contains kernel" : "find kernel");
    }

    template <int B, int G, bool C>
    static int find_wstaged(OaArgs const& a, uint32_t items, void const* keys, void* out, uint32_t n, WaitCtl wc,
                            cudaStream_t s)
    {
        void (*k)(OaArgs, void const*, void*, uint32_t, WaitCtl) = nullptr;
        if (items >= 4 && G >= 4) k = k_find_wstaged<S, B, G, (G >= 4 ? 4 : 1), C>;
        else if (items >= 2) k = k_find_wstaged<S, B, G, 2, C>;
        else k = k_find_wstaged<S, B, G, 1, C>;
        uint64_t warps = (n + kWarpStageKeys - 1) / kWarpStageKeys;
        uint32_t grid = grid_for((void const*)k, kBlock, warps ? warps : 1, kBlock / 32);
        k<<<grid, kBlock, 0, s>>>(a, keys, out, n, wc);
        return check_launch(C ? "contains kernel" : "find kernel");
    }

    template <int B, int G, bool C>
    static int find_wdefer(OaArgs const& a, uint32_t items, void const* keys, void* out, uint32_t n, WaitCtl wc,
                           cudaStream_t s)
    {
        void (*k)(OaArgs, void const*, void*, uint32_t, WaitCtl) = nullptr;
        if (items >= 4 && G >= 4) k = k_find_wdefer<S, B, G, (G >= 4 ? 4 : 1), C>;
        else if (items >= 2) k = k_find_wdefer<S, B, G, 2, C>;
        else k = k_find_wdefer<S, B, G, 1, C>;
        uint64_t warps = (n + kWarpStageKeys - 1) / kWarpStageKeys;
        uint32_t grid = grid_for((void const*)k, kBlock, warps ? warps : 1, kBlock / 32);
        k<<<grid, kBlock, 0, s>>>(a, keys, out, n, wc);
        return check_launch(C ? "contains kernel" : "find kernel");
    }

    template <int B, bool C>
    static int find_bulk(OaArgs const& a, void const* keys, void* out, uint32_t n, WaitCtl wc, cudaStream_t s)
    {
        if constexpr (S::bytes == 16) {
            auto k = k_find_bulk<S, B, C>;
            constexpr uint32_t smem = bulk_window_smem<S, B>();
            // a per-device function attribute: set on every launch (about a microsecond)
            cudaError_t const ea = cudaFuncSetAttribute((void const*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        smem);
            if (ea != cudaSuccess) return cuda_fail(ea, "bulk find attribute");
            int per_sm = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (void const*)k, kBlock, smem);
            if (e != cudaSuccess) return cuda_fail(e, "bulk find occupancy");
            uint64_t chunks = n / kStageKeys;
            uint64_t cap = uint64_t(per_sm < 1 ? 1 : per_sm) * sm_count();
            uint32_t grid = uint32_t(chunks == 0 ? 1 : (chunks < cap ? chunks : cap));
            k<<<grid, kBlock, smem, s>>>(a, keys, out, n, wc);
            return check_launch(C ? "contains kernel" : "find kernel");
        } else {
            return fail(B2CO_EINVAL, "bulk windows need 16-byte slots");
        }
    }

    // The default lookup shapes only (layouts without kAllShapes): per-warp
    // staging with deferred continuations, 2 or 4 lanes per window, one or two
    // windows in flight; the ballot tile (stencils, unaligned key streams) or
    // one lane per key (bucket size 1) otherwise.
    template <int B, bool C>
    static int find_default(OaArgs const& a, uint32_t lanes, uint32_t items, void const* keys,
                            uint8_t const* stencil, void* out, uint32_t n, WaitCtl wc, cudaStream_t s)
    {
        bool const staged = !stencil && (reinterpret_cast<uintptr_t>(keys) & 15) == 0 && n >= kWarpStageKeys &&
                            B > 1 && lanes >= 2;
        uint32_t const q = (items & ~(kShapeDeferred | kShapeWarpStaged | kShapeSegmented | kShapeBulk)) >= 2 ? 2 : 1;
        if (staged) {
            void (*k)(OaArgs, void const*, void*, uint32_t, WaitCtl) = nullptr;
            if (lanes == 2) k = q == 2 ? k_find_wdefer<S, B, 2, 2, C> : k_find_wdefer<S, B, 2, 1, C>;
            else k = q == 2 ? k_find_wdefer<S, B, 4, 2, C> : k_find_wdefer<S, B, 4, 1, C>;
            uint64_t warps = (n + kWarpStageKeys - 1) / kWarpStageKeys;
            k<<<grid_for((void const*)k, kBlock, warps ? warps : 1, kBlock / 32), kBlock, 0, s>>>(a, keys, out, n, wc);
            return check_launch(C ? "contains kernel" : "find kernel");
        }
        void (*k)(OaArgs, void const*, uint8_t const*, void*, uint32_t) = nullptr;
        uint64_t per_block = kBlock;
        if (B == 1 || lanes <= 1) k = k_find_lane<S, B, 1, C>;
        else if (lanes == 2) k = k_find_tile<S, B, 2, C>, per_block /= 2;
        else k = k_find_tile<S, B, 4, C>, per_block /= 4;
        k<<<grid_for((void const*)k, kBlock, n, per_block), kBlock, 0, s>>>(a, keys, stencil, out, n);
        return check_launch(C ? "contains kernel" : "find kernel");
    }

    template <int B, bool C>
    static int find_shape(OaArgs const& a, uint32_t lanes, uint32_t items, void const* keys, uint8_t const* stencil,
                          void* out, uint32_t n, WaitCtl wc, cudaStream_t s)
    {
        if constexpr (!kAllShapes) {
            return find_default<B, C>(a, lanes, items, keys, stencil, out, n, wc, s);
        } else {
            return find_any<B, C>(a, lanes, items, keys, stencil, out, n, wc, s);
        }
    }

    template <int B, bool C>
    static int find_any(OaArgs const& a, uint32_t lanes, uint32_t items, void const* keys, uint8_t const* stencil,
                        void* out, uint32_t n, WaitCtl wc, cudaStream_t s)
    {
        bool const stageable = !stencil && (reinterpret_cast<uintptr_t>(keys) & 15) == 0 && n >= kStageKeys && B > 1;
        // bulk-window path: 16-byte slots only
        if constexpr (B == 5) {  // the block-staged, warp-staged and bulk shapes: bucket size 5 only (build time)
            if ((items & kShapeBulk) && stageable && S::bytes == 16) return find_bulk<B, C>(a, keys, out, n, wc, s);
        } else if (stageable && lanes >= 2) {
            items |= kShapeDeferred;  // other bucket sizes stage keys the default way
        }
        items &= ~kShapeBulk;
        // staged path: no stencil, 16-byte aligned key stream, at least one stage of keys
        bool const staged = stageable && lanes >= 2;
        if (staged && (items & kShapeDeferred)) {
            items &= ~(kShapeDeferred | kShapeWarpStaged | kShapeSegmented);
            if (lanes == 2) return find_wdefer<B, 2, C>(a, items, keys, out, n, wc, s);
            if (lanes == 4) return find_wdefer<B, 4, C>(a, items, keys, out, n, wc, s);
            return find_wdefer<B, 8, C>(a, items, keys, out, n, wc, s);
        }
        items &= ~kShapeDeferred;
        if constexpr (B == 5) {
            if (staged && (items & kShapeWarpStaged)) {
                items &= ~(kShapeWarpStaged | kShapeSegmented);
                if (lanes == 2) return find_wstaged<B, 2, C>(a, items, keys, out, n, wc, s);
                if (lanes == 4) return find_wstaged<B, 4, C>(a, items, keys, out, n, wc, s);
                return find_wstaged<B, 8, C>(a, items, keys, out, n, wc, s);
            }
            items &= ~kShapeWarpStaged;
            if (staged) {
                bool const seg = (items & kShapeSegmented) != 0;
                items &= ~kShapeSegmented;
                if (seg) {
                    if (lanes == 2) return find_staged<B, 2, C, true>(a, items, keys, out, n, wc, s);
                    if (lanes == 4) return find_staged<B, 4, C, true>(a, items, keys, out, n, wc, s);
                    return find_staged<B, 8, C, true>(a, items, keys, out, n, wc, s);
                }
                if (lanes == 2) return find_staged<B, 2, C, false>(a, items, keys, out, n, wc, s);
                if (lanes == 4) return find_staged<B, 4, C, false>(a, items, keys, out, n, wc, s);
                return find_staged<B, 8, C, false>(a, items, keys, out, n, wc, s);
            }
        }
        items &= ~kShapeWarpStaged;
        items &= ~kShapeSegmented;
        void (*k)(OaArgs, void const*, uint8_t const*, void*, uint32_t) = nullptr;
        uint64_t per_block = kBlock;
        if (B == 1 || lanes <= 1) {
            if (items >= 4) k = k_find_lane<S, B, 4, C>, per_block *= 4;
            else if (items == 2) k = k_find_lane<S, B, 2, C>, per_block *= 2;
            else k = k_find_lane<S, B, 1, C>;
        } else if (lanes == 2) {
            k = k_find_tile<S, B, 2, C>, per_block /= 2;
        } else if (lanes == 4) {
            k = k_find_tile<S, B, 4, C>, per_block /= 4;
        } else {
            k = k_find_tile<S, B, 8, C>, per_block /= 8;
        }
        k<<<grid_for((void const*)k, kBlock, n, per_block), kBlock, 0, s>>>(a, keys, stencil, out, n);
        return check_launch(C ? "contains kernel" : "find kernel");
    }

    static int find(OaArgs const& a, uint32_t b, uint32_t lanes, uint32_t items, bool contains, void const* keys,
                    uint8_t const* stencil, void* out, uint32_t n, WaitCtl wc, cudaStream_t s)
    {
        return with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            return contains ? find_shape<B, true>(a, lanes, items, keys, stencil, out, n, wc, s)
                            : find_shape<B, false>(a, lanes, items, keys, stencil, out, n, wc, s);
        });
    }

    static int erase(OaArgs const& a, uint32_t b, void const* keys, uint32_t n, unsigned long long* counters,
                     cudaStream_t s)
    {
        return with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            auto k = k_erase<S, B>;
            k<<<grid_for((void const*)k, kBlock, n, kBlock), kBlock, 0, s>>>(a, keys, n, counters);
            return check_launch("erase kernel");
        });
    }

    static int count(OaArgs const& a, uint32_t b, void const* keys, uint32_t n, unsigned long long* counter,
                     cudaStream_t s)
    {
        return with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            auto k = k_count<S, B>;
            k<<<grid_for((void const*)k, kBlock, n, kBlock), kBlock, 0, s>>>(a, keys, n, counter);
            return check_launch("count kernel");
        });
    }

    static constexpr OaOps ops{&clear, &insert, &assign_if, &iaf_race, &iaf_first, &find, &erase, &count};
};

template <class S>
struct GroupImpl {
    static constexpr uint32_t kBlock = 256;

    // `shape` packs lanes per window (bits 0-7), keys in flight per lane group
    // (bits 8-15; 1 = one key per tile, resolved at once) and threads per block
    // (bits 16-31; 0 = 256).  Keys per tile above 1 run the deferred kernel;
    // its 2-, 4- and 8-lane variants other than 4x2 exist for bucket size 5.
    template <int B, bool C>
    static int find_b(GroupArgs const& g, uint32_t shape, void const* keys, void* out, uint64_t n, cudaStream_t s)
    {
        uint32_t const lanes = shape & 0xffu, items = (shape >> 8) & 0xffu;
        uint32_t const block = (shape >> 16) ? (shape >> 16) : kBlock;
        void (*k)(GroupArgs, void const*, void*, uint64_t) = nullptr;
        if (lanes >= 2 && items >= 2) {
            if constexpr (B == 5) {
                if (lanes == 2) k = k_group_find_q<S, B, 2, 2, C>;
                else if (lanes == 4 && items >= 4) k = k_group_find_q<S, B, 4, 4, C>;
                else if (lanes == 8) k = items >= 4 ? k_group_find_q<S, B, 8, 4, C> : k_group_find_q<S, B, 8, 2, C>;
            }
            if (!k) k = k_group_find_q<S, B, 4, 2, C>;
        } else if (lanes <= 1) {
            k = k_group_find<S, B, 1, C>;
        } else if (lanes == 2) {
            k = k_group_find<S, B, 2, C>;
        } else if (lanes == 4) {
            k = k_group_find<S, B, 4, C>;
        } else {
            k = k_group_find<S, B, 8, C>;
        }
        // persistent: every resident block, spans balanced by items
        k<<<grid_for((void const*)k, block, n, 1), block, 0, s>>>(g, keys, out, n);
        return OaImpl<S>::check_launch(C ? "group contains kernel" : "group find kernel");
    }

    static int find(GroupArgs const& g, uint32_t b, uint32_t shape, bool contains, void const* keys, void* out,
                    uint64_t n, cudaStream_t s)
    {
        return OaImpl<S>::with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            return contains ? find_b<B, true>(g, shape, keys, out, n, s) : find_b<B, false>(g, shape, keys, out, n, s);
        });
    }

    static int insert(GroupArgs const& g, uint32_t b, void const* pairs, uint64_t n, unsigned long long* failed,
                      cudaStream_t s)
    {
        return OaImpl<S>::with_b(b, [&](auto bc) {
            constexpr int B = decltype(bc)::value;
            auto k = k_group_insert<S, B>;
            k<<<grid_for((void const*)k, kBlock, n, 1), kBlock, 0, s>>>(g, pairs, n, failed);
            return OaImpl<S>::check_launch("group insert kernel");
        });
    }

    static constexpr GroupOps ops{&find, &insert};
};

}  // namespace b2co

#define B2CO_DEFINE_OA_OPS(NAME, GNAME, KB, VB)            \
    namespace b2co {                                       \
    OaOps const NAME = OaImpl<SlotT<KB, VB>>::ops;         \
    GroupOps const GNAME = GroupImpl<SlotT<KB, VB>>::ops;  \
    }

// Layouts served by single tables only (no table-group kernels): 2-byte keys
// and floating-point keys (FK = true).
#define B2CO_DEFINE_OA_OPS_ONLY(NAME, KB, VB, FK)          \
    namespace b2co {                                       \
    OaOps const NAME = OaImpl<SlotT<KB, VB, FK>>::ops;     \
    }
