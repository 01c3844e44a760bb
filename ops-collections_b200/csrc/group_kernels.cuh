// group_kernels.cuh -- persistent kernels over a group of independent tables
// (thousands of StaticMaps of uneven sizes in one slab, the batched pattern of
// per-partition group-by / join builds).
//
// One launch covers every table: the items of all tables are concatenated
// (table t owns items [offsets[t], offsets[t+1])) and each warp takes one
// contiguous span of the concatenation, so work is balanced by items, not by
// tables.  A lane finds its table once by binary search and then only walks
// forward; the table's probe parameters stay in registers while it does not
// change.  Per key the algorithms are exactly the single-table ones.
#pragma once

#include "oa_kernels.cuh"

namespace b2co {

struct GroupTable {
    uint64_t slot_offset;  // first slot of the table in the slab
    ProbeParams probe;
};

struct GroupArgs {
    void* slots;
    GroupTable const* tables;
    uint64_t const* offsets;  // count + 1 item offsets (device)
    uint32_t count;
    uint64_t empty_key;
    uint64_t empty_value;
};

__device__ __forceinline__ uint32_t group_table_of(uint64_t const* offsets, uint32_t count, uint64_t i)
{
    uint32_t lo = 0, hi = count;  // offsets[lo] <= i < offsets[hi]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(offsets + mid) <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <class S>
__device__ __forceinline__ OaArgs group_table_args(GroupArgs const& g, uint32_t t)
{
    OaArgs a;
    GroupTable const& d = g.tables[t];
    a.slots = static_cast<typename S::Raw*>(g.slots) + d.slot_offset;
    a.probe = d.probe;
    a.empty_key = g.empty_key;
    a.empty_value = g.empty_value;
    a.erased_key = g.empty_key;
    return a;
}

// Span of the concatenation owned by this warp: multiples of `step` items.
__device__ __forceinline__ void warp_span(uint64_t n, uint32_t step, uint64_t& begin, uint64_t& end)
{
    uint64_t const warps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    uint64_t const warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    uint64_t span = (n + warps - 1) / warps;
    span = (span + step - 1) / step * step;
    begin = warp * span;
    end = begin + span < n ? begin + span : n;
}

// One lane per key: the window is scanned in the lane's own registers, with no
// ballots or shuffles, and a key that needs further windows walks on alone.
template <class S, int B, bool CONTAINS>
__device__ __forceinline__ void group_find_lane(GroupArgs const& g, void const* keys, void* out, uint64_t begin,
                                                uint64_t end)
{
    using Raw = typename S::Raw;
    uint32_t const lane = threadIdx.x & 31;
    uint32_t t = group_table_of(g.offsets, g.count, begin + lane < end ? begin + lane : begin);
    OaArgs a = group_table_args<S>(g, t);
    uint64_t next_off = __ldg(g.offsets + t + 1);
    for (uint64_t i = begin + lane; i < end; i += 32) {
        if (i >= next_off) {
            do {
                ++t;
                next_off = __ldg(g.offsets + t + 1);
            } while (i >= next_off);
            a = group_table_args<S>(g, t);
        }
        uint64_t const key = uint64_t(__ldg(reinterpret_cast<typename Io<S>::Key const*>(keys) + i));
        uint32_t const init = probe_init<S::key_bytes, B>(a.probe, key);
        Raw w[B];
        load_window<S, B>(reinterpret_cast<Raw const*>(a.slots), init, w);
        Raw stop;
        uint64_t payload = empty_payload<S>(a);
        bool hit;
        if (scan_window<S, B>(w, key, a.empty_key, stop)) {
            hit = S::key(stop) != a.empty_key;
            if (hit) payload = S::value(stop);
        } else {
            hit = find_rest<S, B>(a, key, init, payload);
        }
        if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = hit;
        else reinterpret_cast<typename Io<S>::Payload*>(out)[i] = typename Io<S>::Payload(hit ? payload : empty_payload<S>(a));
    }
}

template <class S, int B, int G, bool CONTAINS>
__global__ void __launch_bounds__(256) k_group_find(GroupArgs g, void const* keys, void* out, uint64_t n)
{
    if constexpr (G == 1) {
        uint64_t begin, end;
        warp_span(n, 32, begin, end);
        if (begin < end) group_find_lane<S, B, CONTAINS>(g, keys, out, begin, end);
        return;
    }
    using Raw = typename S::Raw;
    constexpr int ROUNDS = (B + G - 1) / G;
    constexpr uint32_t TILES = 32 / G;
    uint32_t const lane = threadIdx.x & 31, r = lane % G, tile_lane0 = lane & ~uint32_t(G - 1), tile = lane / G;
    uint64_t begin, end;
    warp_span(n, TILES, begin, end);
    if (begin >= end) return;  // warp-uniform
    uint32_t t = group_table_of(g.offsets, g.count, begin + tile < end ? begin + tile : begin);
    OaArgs a = group_table_args<S>(g, t);
    uint64_t next_off = __ldg(g.offsets + t + 1);
    for (uint64_t i0 = begin; i0 < end; i0 += TILES) {
        uint64_t const i = i0 + tile;
        bool const live = i < end;
        if (live && i >= next_off) {
            do {
                ++t;
                next_off = __ldg(g.offsets + t + 1);
            } while (i >= next_off);
            a = group_table_args<S>(g, t);
        }
        uint64_t const key = live ? uint64_t(__ldg(reinterpret_cast<typename Io<S>::Key const*>(keys) + i)) : 0;
        uint32_t const init = live ? probe_init<S::key_bytes, B>(a.probe, key) : 0;
        Raw const* slots = reinterpret_cast<Raw const*>(a.slots);
        Raw w[ROUNDS];
        if (live) {
#pragma unroll
            for (int k = 0; k < ROUNDS; ++k)
                if (int(r) + k * G < B) w[k] = ld_ro(slots + init + r + k * G);
        }
        TileResult res{0, false, !live};
        tile_resolve<S, B, G, ROUNDS>(a, w, key, r, tile_lane0, !live, res);
        if (__any_sync(0xffffffffu, !res.done)) res = tile_continue<S, B, G, ROUNDS>(a, slots, key, init, r, tile_lane0, res);
        if (r == 0 && live) {
            if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[i] = res.hit;
            else reinterpret_cast<typename Io<S>::Payload*>(out)[i] =
                typename Io<S>::Payload(res.hit ? res.payload : empty_payload<S>(a));
        }
    }
}

// The group lookup in the single-table default's shape: G lanes share a
// window, each tile keeps Q keys in flight, and a key whose first window
// settles nothing is queued in the warp's shared-memory ring with its table
// and followed a pass at a time (a pass waits on one window load).  Each
// q-slot of a tile walks forward through the tables on its own, so a pass may
// span a table boundary.  Blocks of up to 256 threads.
template <class S, int B, int G, int Q, bool CONTAINS>
__global__ void __launch_bounds__(256) k_group_find_q(GroupArgs g, void const* keys, void* out, uint64_t n)
{
    static_assert(Q <= G && G >= 2 && G <= 8, "tile shape");
    using Raw = typename S::Raw;
    constexpr int ROUNDS = (B + G - 1) / G;
    constexpr uint32_t TILES = 32 / G;
    constexpr uint32_t PASS = TILES * Q;
    static_assert(2 * PASS <= kDeferRing, "the ring must hold a pass on top of a partial one");
    constexpr uint32_t RING = kDeferRing - 1;
    __shared__ uint64_t qkey[8][kDeferRing], qpos[8][kDeferRing];
    __shared__ uint32_t qtab[8][kDeferRing], qinit[8][kDeferRing], qidx[8][kDeferRing];

    uint32_t const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t const r = lane % G, tile_lane0 = lane & ~uint32_t(G - 1), tile = lane / G;
    uint64_t begin, end;
    warp_span(n, PASS, begin, end);
    if (begin >= end) return;  // warp-uniform
    uint32_t head = 0, count = 0;
    using Key = typename Io<S>::Key;
    Key const* kin = static_cast<Key const*>(keys);

    auto write = [&](uint64_t pos, bool hit, Raw const& slot, uint64_t empty) {
        if constexpr (CONTAINS) reinterpret_cast<uint8_t*>(out)[pos] = hit;
        else reinterpret_cast<typename Io<S>::Payload*>(out)[pos] = typename Io<S>::Payload(hit ? S::value(slot) : empty);
    };
    auto enqueue = [&](bool unsettled, uint64_t key, uint32_t tab, uint32_t init, uint32_t idx, uint64_t pos) {
        uint32_t const m = __ballot_sync(0xffffffffu, unsettled);
        if (unsettled) {
            uint32_t const e = (head + count + __popc(m & ((1u << lane) - 1u))) & RING;
            qkey[warp][e] = key;
            qtab[warp][e] = tab;
            qinit[warp][e] = init;
            qidx[warp][e] = idx;
            qpos[warp][e] = pos;
        }
        count += __popc(m);
    };
    uint64_t const empty = S::is_set ? g.empty_key : g.empty_value;
    auto follow = [&]() {
        __syncwarp();
        uint32_t const take = count < PASS ? count : PASS;
        uint64_t key[Q], pos[Q];
        uint32_t tab[Q], init[Q], idx[Q];
        bool live[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint32_t const j = q * TILES + tile;
            live[q] = j < take;
            uint32_t const e = (head + (live[q] ? j : 0u)) & RING;
            key[q] = qkey[warp][e];
            tab[q] = qtab[warp][e];
            init[q] = qinit[warp][e];
            idx[q] = qidx[warp][e];
            pos[q] = qpos[warp][e];
        }
        __syncwarp();
        head = (head + take) & RING;
        count -= take;
        Raw w[Q][ROUNDS];
        Raw const* base[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            GroupTable const& T = g.tables[live[q] ? tab[q] : 0u];
            base[q] = static_cast<Raw const*>(g.slots) + T.slot_offset;
            if (live[q]) {
                idx[q] = probe_next(idx[q], probe_step<S::key_bytes, B>(T.probe, key[q]), T.probe.capacity);
                if (idx[q] == init[q]) {  // a whole cycle: not present
                    if (r == 0) write(pos[q], false, Raw{}, empty);
                    live[q] = false;
                }
            }
            load_range<S, B, G, ROUNDS>(base[q], idx[q], 0, B, r, !live[q], w[q]);
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int own;
            Raw mine{};
            int const st = tile_first_stop<S, B, G, ROUNDS>(w[q], !live[q], key[q], g.empty_key, r, own, mine);
            if (live[q] && st != kNoStop && own == st) write(pos[q], S::key(mine) != g.empty_key, mine, empty);
            enqueue(live[q] && st == kNoStop && r == 0, key[q], tab[q], init[q], idx[q], pos[q]);
        }
    };

    uint32_t tq[Q];
    uint64_t nextq[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        uint64_t const i = begin + q * TILES + tile;
        tq[q] = group_table_of(g.offsets, g.count, i < end ? i : end - 1);
        nextq[q] = __ldg(g.offsets + tq[q] + 1);
    }
    for (uint64_t i0 = begin; i0 < end; i0 += PASS) {
        uint64_t key[Q];
        uint32_t idx[Q];
        bool live[Q];
        uint32_t my_init = 0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            uint64_t const i = i0 + q * TILES + tile;
            live[q] = i < end;
            if (live[q] && i >= nextq[q]) {
                do {
                    ++tq[q];
                    nextq[q] = __ldg(g.offsets + tq[q] + 1);
                } while (i >= nextq[q]);
            }
            key[q] = live[q] ? uint64_t(__ldg(kin + i)) : 0;
            if (int(r) == q && live[q]) my_init = probe_init<S::key_bytes, B>(g.tables[tq[q]].probe, key[q]);
        }
        Raw w[Q][ROUNDS];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            idx[q] = __shfl_sync(0xffffffffu, my_init, tile_lane0 + q);
            Raw const* base = static_cast<Raw const*>(g.slots) + g.tables[tq[q]].slot_offset;
            load_range<S, B, G, ROUNDS>(base, idx[q], 0, B, r, !live[q], w[q]);
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int own;
            Raw mine{};
            uint64_t const i = i0 + q * TILES + tile;
            int const st = tile_first_stop<S, B, G, ROUNDS>(w[q], !live[q], key[q], g.empty_key, r, own, mine);
            if (live[q] && st != kNoStop && own == st) write(i, S::key(mine) != g.empty_key, mine, empty);
            enqueue(live[q] && st == kNoStop && r == 0, key[q], tq[q], idx[q], idx[q], i);
        }
        while (count >= PASS) follow();
    }
    while (count > 0) follow();
}

template <class S, int B>
__global__ void __launch_bounds__(256) k_group_insert(GroupArgs g, void const* pairs, uint64_t n,
                                                      unsigned long long* failed_counter)
{
    uint64_t begin, end;
    warp_span(n, 32, begin, end);
    uint32_t failed = 0;
    if (begin < end) {
        uint32_t const lane = threadIdx.x & 31;
        uint32_t t = group_table_of(g.offsets, g.count, begin + lane < end ? begin + lane : begin);
        OaArgs a = group_table_args<S>(g, t);
        uint64_t next_off = __ldg(g.offsets + t + 1);
        for (uint64_t i0 = begin; i0 < end; i0 += 32) {
            uint64_t const i = i0 + lane;
            if (i >= end) continue;
            if (i >= next_off) {
                do {
                    ++t;
                    next_off = __ldg(g.offsets + t + 1);
                } while (i >= next_off);
                a = group_table_args<S>(g, t);
            }
            typename S::Raw p = ld_ro(reinterpret_cast<typename S::Raw const*>(pairs) + i);
            failed += insert_one<S, B, false>(a, S::key(p), S::value(p)) != kSuccess;
        }
    }
    if (failed_counter) warp_add_counter(failed_counter, failed);
}

}  // namespace b2co
