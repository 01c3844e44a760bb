// multi.cu -- StaticMultiset<Key> and StaticMultimap<Key, Value> (Key, Value
// int32 or int64) for B200.  The reference's containers expose no slot layout,
// so the storage here is designed for the GPU, and only the observable rules
// follow the reference (include/static_multiset.h, include/static_multimap.h,
// static_multimap_ref.h):
//
// StaticMultiset: an `ordered` array of the accepted keys in insertion order
// (RetrieveAll) plus a key -> count table (multi_common.cuh) sized for the
// capacity.  Insert ranks the valid selected keys in input order with a
// device-wide scan, keeps the first (capacity - size), appends them and adds 1
// to each key's count; every query is one table probe.
//
// StaticMultimap: a dense pair array in accepted insertion order
// (RetrieveAll) plus, built lazily at the first query after an insert, a
// grouped index: the key -> count table, an exclusive scan of the counts into
// per-key offsets, and a CSR array of every key's values in ascending order,
// produced by a stable LSD radix sort of (value, table slot) records.  Find is
// then the first value of the key's run (its minimum), Count its length and
// Retrieve a copy of the run -- no per-query sorting.
#include <algorithm>
#include <new>

#include "multi_common.cuh"

using namespace b2co;
using namespace b2co::multi;

namespace {

constexpr uint64_t kMaxElements = 1ull << 31;

cudaStream_t cs(b2co_stream s) { return reinterpret_cast<cudaStream_t>(s); }

uint64_t mask_bits(uint64_t v, uint32_t bytes) { return bytes >= 8 ? v : (v & ((1ull << (8 * bytes)) - 1)); }

// Device scratch grown on demand.
struct Scratch {
    void* p = nullptr;
    uint64_t bytes = 0;
    int reserve(uint64_t need)
    {
        if (need <= bytes) return B2CO_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, need);
        if (e != cudaSuccess) return cuda_fail(e, "multi-container scratch");
        bytes = need;
        return B2CO_OK;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

int read_word(uint64_t const* dev, uint64_t* host_pinned, cudaStream_t s, uint64_t* out)
{
    B2CO_CUDA(cudaMemcpyAsync(host_pinned, dev, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    B2CO_CUDA(cudaStreamSynchronize(s));
    *out = *host_pinned;
    return B2CO_OK;
}

template <class F, class A>
int apply_scanned(F f, A act, uint64_t n, uint64_t const* tile_offsets, cudaStream_t s)
{
    if (n == 0) return B2CO_OK;
    k_tile_apply<<<uint32_t((n + kTile - 1) / kTile), kThreads, 0, s>>>(f, act, n, tile_offsets);
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

// ---------------------------------------------------------------------------
// StaticMultiset
// ---------------------------------------------------------------------------

template <int KB>
struct MsetFlag {  // a valid selected key -> 1, a selected sentinel key -> 2^32
    KeyWord<KB> const* keys;
    uint8_t const* stencil;
    KeyWord<KB> empty;
    __device__ uint64_t operator()(uint64_t i) const
    {
        if (stencil && !stencil[i]) return 0;
        return keys[i] == empty ? (1ull << 32) : 1ull;
    }
};

template <int KB>
struct MsetAppend {
    KeyTable<KB> t;
    KeyWord<KB> const* keys;
    KeyWord<KB>* ordered;
    uint64_t size, accepted;
    __device__ void operator()(uint64_t i, uint64_t v, uint64_t prefix) const
    {
        if (v != 1) return;
        uint64_t const rank = prefix & 0xffffffffull;
        if (rank >= accepted) return;
        ordered[size + rank] = keys[i];
        table_add<KB>(t, keys[i], 1u);
    }
};

template <int KB>
struct MsetCount {
    KeyTable<KB> t;
    KeyWord<KB> const* keys;
    __device__ uint64_t operator()(uint64_t i) const
    {
        uint64_t const s = table_find<KB>(t, keys[i]);
        return s == ~0ull ? 0 : t.counts[s];
    }
};

template <int KB>
struct MsetRetrieve {
    KeyWord<KB> const* keys;
    KeyWord<KB>* probe_out;
    KeyWord<KB>* match_out;
    __device__ void operator()(uint64_t i, uint64_t count, uint64_t offset) const
    {
        KeyWord<KB> const k = keys[i];
        for (uint64_t j = 0; j < count; ++j) {
            probe_out[offset + j] = k;
            match_out[offset + j] = k;
        }
    }
};

// mode: 0 contains (u8), 1 find (key), 2 count each (u64), 3 count each, 0 -> 1 (u64)
template <int KB, int MODE>
__global__ void __launch_bounds__(256) k_mset_query(KeyTable<KB> t, KeyWord<KB> const* keys, uint8_t const* stencil,
                                                    void* out, uint64_t n)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        bool const sel = !stencil || stencil[i];
        KeyWord<KB> const k = keys[i];
        uint64_t c = 0;
        if (sel) {
            uint64_t const s = table_find<KB>(t, k);
            c = s == ~0ull ? 0 : t.counts[s];
        }
        if constexpr (MODE == 0) static_cast<uint8_t*>(out)[i] = c > 0;
        else if constexpr (MODE == 1) static_cast<KeyWord<KB>*>(out)[i] = c > 0 ? k : t.empty;
        else if constexpr (MODE == 2) static_cast<unsigned long long*>(out)[i] = c;
        else static_cast<unsigned long long*>(out)[i] = c ? c : 1;
    }
}

// ---------------------------------------------------------------------------
// StaticMultimap
// ---------------------------------------------------------------------------

template <int VB>
__device__ __forceinline__ unsigned long long order_bits(uint64_t v)
{
    if constexpr (VB == 4) return (v & 0xffffffffull) ^ 0x80000000ull;
    else return v ^ 0x8000000000000000ull;
}
template <int VB>
__device__ __forceinline__ uint64_t from_order_bits(unsigned long long b)
{
    if constexpr (VB == 4) return (b ^ 0x80000000ull) & 0xffffffffull;
    else return b ^ 0x8000000000000000ull;
}

template <int KB, int VB>
struct MmapSelect {
    uint8_t const* stencil;
    __device__ uint64_t operator()(uint64_t i) const { return !stencil || stencil[i] ? 1 : 0; }
};

template <int KB, int VB>
__global__ void __launch_bounds__(256) k_mmap_validate(typename SlotT<KB, VB>::Raw const* pairs, uint8_t const* stencil,
                                                       uint64_t n, uint64_t ek, uint64_t ev, unsigned int* status)
{
    using S = SlotT<KB, VB>;
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    bool bad = false;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (stencil && !stencil[i]) continue;
        typename S::Raw const r = pairs[i];
        bad |= S::key(r) == ek || S::value(r) == ev;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, 1u);
}

template <int KB, int VB>
struct MmapAppend {
    typename SlotT<KB, VB>::Raw const* pairs;
    typename SlotT<KB, VB>::Raw* dense;
    uint64_t size, accepted;
    __device__ void operator()(uint64_t i, uint64_t v, uint64_t rank) const
    {
        using S = SlotT<KB, VB>;
        if (!v || rank >= accepted) return;
        typename S::Raw const r = pairs[i];
        dense[size + rank] = S::make(S::key(r), S::value(r));  // padding bytes normalized
    }
};

template <int KB, int VB>
__global__ void __launch_bounds__(256) k_mmap_records(KeyTable<KB> t, typename SlotT<KB, VB>::Raw const* dense,
                                                      uint64_t n, Record* rec)
{
    using S = SlotT<KB, VB>;
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        typename S::Raw const r = dense[i];
        uint64_t const slot = table_add<KB>(t, KeyWord<KB>(S::key(r)), 1u);
        Record x;
        x.vbits = order_bits<VB>(S::value(r));
        x.slot = uint32_t(slot);
        x.pad = 0;
        rec[i] = x;
    }
}

struct CountOf {
    uint32_t const* counts;
    __device__ uint64_t operator()(uint64_t i) const { return counts[i]; }
};
struct WriteOffset {
    uint32_t* offsets;
    __device__ void operator()(uint64_t i, uint64_t, uint64_t prefix) const { offsets[i] = uint32_t(prefix); }
};
struct HistOf {
    uint64_t* h;
    __device__ uint64_t operator()(uint64_t i) const { return h[i]; }
};
struct HistPrefix {
    uint64_t* h;
    __device__ void operator()(uint64_t i, uint64_t, uint64_t prefix) const { h[i] = prefix; }
};

template <int VB>
__global__ void __launch_bounds__(256) k_mmap_csr(Record const* rec, uint64_t n, void* csr)
{
    using V = typename std::conditional<VB == 4, unsigned int, unsigned long long>::type;
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        static_cast<V*>(csr)[i] = V(from_order_bits<VB>(rec[i].vbits));
}

// mode: 0 contains (u8), 1 find (smallest value or the empty value)
template <int KB, int VB, int MODE>
__global__ void __launch_bounds__(256) k_mmap_query(KeyTable<KB> t, void const* csr, KeyWord<KB> const* keys,
                                                    uint8_t const* stencil, void* out, uint64_t n, uint64_t ev)
{
    using V = typename std::conditional<VB == 4, unsigned int, unsigned long long>::type;
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint64_t s = ~0ull;
        if (!stencil || stencil[i]) s = table_find<KB>(t, keys[i]);
        if constexpr (MODE == 0) static_cast<uint8_t*>(out)[i] = s != ~0ull;
        else static_cast<V*>(out)[i] = s == ~0ull ? V(ev) : static_cast<V const*>(csr)[t.offsets[s]];
    }
}

template <int KB>
struct MmapCount {
    KeyTable<KB> t;
    KeyWord<KB> const* keys;
    __device__ uint64_t operator()(uint64_t i) const
    {
        uint64_t const s = table_find<KB>(t, keys[i]);
        return s == ~0ull ? 0 : t.counts[s];
    }
};

template <int KB, int VB>
struct MmapRetrieve {
    KeyTable<KB> t;
    KeyWord<KB> const* keys;
    void const* csr;
    KeyWord<KB>* key_out;
    void* value_out;
    __device__ void operator()(uint64_t i, uint64_t count, uint64_t offset) const
    {
        using V = typename std::conditional<VB == 4, unsigned int, unsigned long long>::type;
        if (!count) return;
        KeyWord<KB> const k = keys[i];
        uint64_t const first = t.offsets[table_find<KB>(t, k)];
        for (uint64_t j = 0; j < count; ++j) {
            key_out[offset + j] = k;
            static_cast<V*>(value_out)[offset + j] = static_cast<V const*>(csr)[first + j];
        }
    }
};

template <int KB, int VB>
__global__ void __launch_bounds__(256) k_mmap_export(typename SlotT<KB, VB>::Raw const* dense, uint64_t n,
                                                     KeyWord<KB>* key_out, void* value_out)
{
    using S = SlotT<KB, VB>;
    using V = typename std::conditional<VB == 4, unsigned int, unsigned long long>::type;
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        typename S::Raw const r = dense[i];
        key_out[i] = KeyWord<KB>(S::key(r));
        static_cast<V*>(value_out)[i] = V(S::value(r));
    }
}

uint32_t blocks_for(uint64_t n) { return uint32_t(std::min<uint64_t>((n + 255) / 256, 148ull * 16)); }

}  // namespace

// ---------------------------------------------------------------------------
// containers
// ---------------------------------------------------------------------------

struct b2co_mset {
    uint64_t capacity = 0, size = 0;
    uint32_t kb = 0;
    uint64_t empty = 0;
    void* ordered = nullptr;
    void* tkeys = nullptr;
    uint32_t* tcounts = nullptr;
    uint64_t tsize = 0;
    Scratch scratch;
    uint64_t* h_word = nullptr;  // pinned

    template <int KB>
    KeyTable<KB> table() const
    {
        return KeyTable<KB>{static_cast<KeyWord<KB>*>(tkeys), tcounts, nullptr, tsize - 1, KeyWord<KB>(empty)};
    }
};

struct b2co_mmap {
    uint64_t capacity = 0, size = 0;
    uint32_t kb = 0, vb = 0;
    uint64_t ek = 0, ev = 0;
    void* dense = nullptr;
    bool dirty = false;
    // grouped index
    void* tkeys = nullptr;
    uint32_t* tcounts = nullptr;
    uint32_t* toffsets = nullptr;
    uint64_t tsize = 0, tsize_alloc = 0;
    Record* rec[2] = {nullptr, nullptr};
    void* csr = nullptr;
    uint64_t rec_cap = 0;
    Scratch scratch, hist;
    unsigned int* d_status = nullptr;
    uint64_t* h_word = nullptr;

    template <int KB>
    KeyTable<KB> table() const
    {
        return KeyTable<KB>{static_cast<KeyWord<KB>*>(tkeys), tcounts, toffsets, tsize - 1, KeyWord<KB>(ek)};
    }
    uint32_t slot_bytes() const { return (kb == 4 && vb == 4) ? 8 : 16; }
};

namespace {

int check_mset(b2co_mset const* s)
{
    if (!s || !s->ordered) return fail(B2CO_ELOGIC, "StaticMultiset: moved-from or destroyed object");
    return B2CO_OK;
}
int check_mmap(b2co_mmap const* m)
{
    if (!m || !m->dense) return fail(B2CO_ELOGIC, "StaticMultimap: moved-from or destroyed object");
    return B2CO_OK;
}

template <int KB>
int mset_clear(b2co_mset* s, cudaStream_t st)
{
    k_table_clear<KB><<<blocks_for(s->tsize), 256, 0, st>>>(s->table<KB>());
    B2CO_CUDA(cudaGetLastError());
    B2CO_CUDA(cudaStreamSynchronize(st));
    s->size = 0;
    return B2CO_OK;
}

template <int KB>
int mset_insert(b2co_mset* s, void const* keys, uint8_t const* stencil, uint64_t n, cudaStream_t st, uint64_t* failed)
{
    if (int e = s->scratch.reserve(scan_scratch_words(n) * 8)) return e;
    uint64_t* sc = s->scratch.as<uint64_t>();
    MsetFlag<KB> f{static_cast<KeyWord<KB> const*>(keys), stencil, KeyWord<KB>(s->empty)};
    if (int e = tile_scan(f, NoAct{}, n, sc, false, st)) return e;
    uint64_t total = 0;
    if (int e = read_word(sc + (n + kTile - 1) / kTile, s->h_word, st, &total)) return e;
    uint64_t const valid = total & 0xffffffffull, invalid = total >> 32;
    uint64_t const accepted = std::min(valid, s->capacity - s->size);
    if (accepted) {
        MsetAppend<KB> act{s->table<KB>(), static_cast<KeyWord<KB> const*>(keys),
                           static_cast<KeyWord<KB>*>(s->ordered), s->size, accepted};
        if (int e = apply_scanned(f, act, n, sc, st)) return e;
        B2CO_CUDA(cudaStreamSynchronize(st));
    }
    s->size += accepted;
    if (failed) *failed = valid - accepted + invalid;
    return B2CO_OK;
}

template <int KB, int MODE>
int mset_query(b2co_mset* s, void const* keys, uint8_t const* stencil, void* out, uint64_t n, cudaStream_t st)
{
    k_mset_query<KB, MODE><<<blocks_for(n), 256, 0, st>>>(s->table<KB>(), static_cast<KeyWord<KB> const*>(keys),
                                                           stencil, out, n);
    B2CO_CUDA(cudaGetLastError());
    B2CO_CUDA(cudaStreamSynchronize(st));
    return B2CO_OK;
}

template <int KB>
int mset_count(b2co_mset* s, void const* keys, uint64_t n, cudaStream_t st, uint64_t* total, bool retrieve,
               void* probe_out, void* match_out, uint64_t cap)
{
    if (int e = s->scratch.reserve(scan_scratch_words(n) * 8)) return e;
    uint64_t* sc = s->scratch.as<uint64_t>();
    MsetCount<KB> f{s->table<KB>(), static_cast<KeyWord<KB> const*>(keys)};
    if (int e = tile_scan(f, NoAct{}, n, sc, false, st)) return e;
    if (int e = read_word(sc + (n + kTile - 1) / kTile, s->h_word, st, total)) return e;
    if (!retrieve || *total == 0) return B2CO_OK;
    if (*total > cap) return fail(B2CO_ERANGE, "StaticMultiset: output capacity too small");
    if (!probe_out || !match_out) return fail(B2CO_EINVAL, "StaticMultiset: null output for a nonempty result");
    MsetRetrieve<KB> act{static_cast<KeyWord<KB> const*>(keys), static_cast<KeyWord<KB>*>(probe_out),
                         static_cast<KeyWord<KB>*>(match_out)};
    if (int e = apply_scanned(f, act, n, sc, st)) return e;
    B2CO_CUDA(cudaStreamSynchronize(st));
    return B2CO_OK;
}

// ---- multimap ------------------------------------------------------------------

template <int KB, int VB>
int mmap_insert(b2co_mmap* m, void const* pairs, uint8_t const* stencil, uint64_t n, cudaStream_t st,
                uint64_t* failed)
{
    using Raw = typename SlotT<KB, VB>::Raw;
    B2CO_CUDA(cudaMemsetAsync(m->d_status, 0, sizeof(unsigned int), st));
    k_mmap_validate<KB, VB><<<blocks_for(n), 256, 0, st>>>(static_cast<Raw const*>(pairs), stencil, n, m->ek, m->ev,
                                                           m->d_status);
    B2CO_CUDA(cudaGetLastError());
    if (int e = m->scratch.reserve(scan_scratch_words(n) * 8)) return e;
    uint64_t* sc = m->scratch.as<uint64_t>();
    MmapSelect<KB, VB> f{stencil};
    if (int e = tile_scan(f, NoAct{}, n, sc, false, st)) return e;
    unsigned int bad = 0;
    B2CO_CUDA(cudaMemcpyAsync(&bad, m->d_status, sizeof(bad), cudaMemcpyDeviceToHost, st));
    uint64_t selected = 0;
    if (int e = read_word(sc + (n + kTile - 1) / kTile, m->h_word, st, &selected)) return e;
    if (bad) return fail(B2CO_EINVAL, "StaticMultimap: selected input contains a reserved key or value");
    uint64_t const accepted = std::min(selected, m->capacity - m->size);
    if (accepted) {
        MmapAppend<KB, VB> act{static_cast<Raw const*>(pairs), static_cast<Raw*>(m->dense), m->size, accepted};
        if (int e = apply_scanned(f, act, n, sc, st)) return e;
        B2CO_CUDA(cudaStreamSynchronize(st));
        m->dirty = true;
    }
    m->size += accepted;
    if (failed) *failed = selected - accepted;
    return B2CO_OK;
}

int mmap_reserve_index(b2co_mmap* m, uint64_t tsize)
{
    if (tsize > m->tsize_alloc) {
        cudaFree(m->tkeys);
        cudaFree(m->tcounts);
        cudaFree(m->toffsets);
        m->tkeys = m->tcounts = m->toffsets = nullptr;
        m->tsize_alloc = 0;
        B2CO_CUDA(cudaMalloc(&m->tkeys, tsize * m->kb));
        B2CO_CUDA(cudaMalloc(reinterpret_cast<void**>(&m->tcounts), tsize * 4));
        B2CO_CUDA(cudaMalloc(reinterpret_cast<void**>(&m->toffsets), tsize * 4));
        m->tsize_alloc = tsize;
    }
    m->tsize = tsize;
    if (m->size > m->rec_cap) {
        cudaFree(m->rec[0]);
        cudaFree(m->rec[1]);
        cudaFree(m->csr);
        m->rec[0] = m->rec[1] = nullptr;
        m->csr = nullptr;
        m->rec_cap = 0;
        B2CO_CUDA(cudaMalloc(reinterpret_cast<void**>(&m->rec[0]), m->size * sizeof(Record)));
        B2CO_CUDA(cudaMalloc(reinterpret_cast<void**>(&m->rec[1]), m->size * sizeof(Record)));
        B2CO_CUDA(cudaMalloc(&m->csr, m->size * m->vb));
        m->rec_cap = m->size;
    }
    return B2CO_OK;
}

// Builds the grouped index of the stored pairs: table of distinct keys with
// counts, per-key offsets, and the values of every key ascending (CSR).
template <int KB, int VB>
int mmap_build(b2co_mmap* m, cudaStream_t st)
{
    if (!m->dirty) return B2CO_OK;
    uint64_t const n = m->size;
    if (int e = mmap_reserve_index(m, table_size_for(n))) return e;
    KeyTable<KB> t = m->table<KB>();
    k_table_clear<KB><<<blocks_for(m->tsize), 256, 0, st>>>(t);
    B2CO_CUDA(cudaGetLastError());
    if (n == 0) {  // an empty table answers every query with a miss
        B2CO_CUDA(cudaStreamSynchronize(st));
        m->dirty = false;
        return B2CO_OK;
    }
    using Raw = typename SlotT<KB, VB>::Raw;
    k_mmap_records<KB, VB><<<blocks_for(n), 256, 0, st>>>(t, static_cast<Raw const*>(m->dense), n, m->rec[0]);
    B2CO_CUDA(cudaGetLastError());
    // per-key offsets: exclusive scan of the counts in slot order
    if (int e = m->scratch.reserve(scan_scratch_words(std::max(m->tsize, uint64_t(256) * ((n + kSortTile - 1) /
                                                                                        kSortTile))) * 8))
        return e;
    uint64_t* sc = m->scratch.as<uint64_t>();
    if (int e = tile_scan(CountOf{m->tcounts}, WriteOffset{m->toffsets}, m->tsize, sc, true, st)) return e;
    // stable LSD radix sort of (value, slot) records: value bytes first, then slot bytes
    uint64_t const ntiles = (n + kSortTile - 1) / kSortTile;
    if (int e = m->hist.reserve(256 * ntiles * 8)) return e;
    uint64_t* h = m->hist.as<uint64_t>();
    int slot_bytes = 0;
    for (uint64_t v = m->tsize - 1; v; v >>= 8) ++slot_bytes;
    int const passes = VB + slot_bytes;
    int cur = 0;
    for (int p = 0; p < passes; ++p) {
        k_radix_hist<<<uint32_t(ntiles), kSortThreads, 0, st>>>(m->rec[cur], n, p, VB, ntiles, h);
        if (int e = tile_scan(HistOf{h}, HistPrefix{h}, 256 * ntiles, sc, true, st)) return e;
        k_radix_scatter<<<uint32_t(ntiles), kSortThreads, 0, st>>>(m->rec[cur], m->rec[1 - cur], n, p, VB, ntiles, h);
        B2CO_CUDA(cudaGetLastError());
        cur = 1 - cur;
    }
    k_mmap_csr<VB><<<blocks_for(n), 256, 0, st>>>(m->rec[cur], n, m->csr);
    B2CO_CUDA(cudaGetLastError());
    B2CO_CUDA(cudaStreamSynchronize(st));
    m->dirty = false;
    return B2CO_OK;
}

template <int KB, int VB, int MODE>
int mmap_query(b2co_mmap* m, void const* keys, uint8_t const* stencil, void* out, uint64_t n, cudaStream_t st)
{
    if (int e = mmap_build<KB, VB>(m, st)) return e;
    k_mmap_query<KB, VB, MODE><<<blocks_for(n), 256, 0, st>>>(m->table<KB>(), m->csr,
                                                               static_cast<KeyWord<KB> const*>(keys), stencil, out, n,
                                                               m->ev);
    B2CO_CUDA(cudaGetLastError());
    B2CO_CUDA(cudaStreamSynchronize(st));
    return B2CO_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

namespace {

template <class F>
int by_kb(uint32_t kb, F f)
{
    return kb == 4 ? f(std::integral_constant<int, 4>{}) : f(std::integral_constant<int, 8>{});
}
template <class F>
int by_kv(uint32_t kb, uint32_t vb, F f)
{
    if (kb == 4) return vb == 4 ? f(std::integral_constant<int, 4>{}, std::integral_constant<int, 4>{})
                                : f(std::integral_constant<int, 4>{}, std::integral_constant<int, 8>{});
    return vb == 4 ? f(std::integral_constant<int, 8>{}, std::integral_constant<int, 4>{})
                   : f(std::integral_constant<int, 8>{}, std::integral_constant<int, 8>{});
}

int check_batch(uint64_t n)
{
    if (n > kMaxBatch) return fail(B2CO_ERANGE, "batch exceeds the 32-bit index range");
    return B2CO_OK;
}

int mset_query_any(b2co_mset* s, void const* keys, uint8_t const* stencil, bool use_stencil, void* out, uint64_t n,
                   b2co_stream st, int mode)
{
    if (int e = check_mset(s)) return e;
    if (n == 0) return B2CO_OK;
    if (!keys || !out) return fail(B2CO_EINVAL, "StaticMultiset: null nonempty buffer");
    if (use_stencil && !stencil) return fail(B2CO_EINVAL, "StaticMultiset: null stencil");
    if (int e = check_batch(n)) return e;
    return by_kb(s->kb, [&](auto k) {
        constexpr int KB = decltype(k)::value;
        switch (mode) {
            case 0: return mset_query<KB, 0>(s, keys, stencil, out, n, cs(st));
            case 1: return mset_query<KB, 1>(s, keys, stencil, out, n, cs(st));
            case 2: return mset_query<KB, 2>(s, keys, stencil, out, n, cs(st));
            default: return mset_query<KB, 3>(s, keys, stencil, out, n, cs(st));
        }
    });
}

int mmap_query_any(b2co_mmap* m, void const* keys, uint8_t const* stencil, bool use_stencil, void* out, uint64_t n,
                   b2co_stream st, int mode)
{
    if (int e = check_mmap(m)) return e;
    if (n == 0) return B2CO_OK;
    if (!keys || !out) return fail(B2CO_EINVAL, "StaticMultimap: null nonempty buffer");
    if (use_stencil && !stencil) return fail(B2CO_EINVAL, "StaticMultimap: null stencil");
    if (int e = check_batch(n)) return e;
    return by_kv(m->kb, m->vb, [&](auto k, auto v) {
        constexpr int KB = decltype(k)::value, VB = decltype(v)::value;
        return mode == 0 ? mmap_query<KB, VB, 0>(m, keys, stencil, out, n, cs(st))
                         : mmap_query<KB, VB, 1>(m, keys, stencil, out, n, cs(st));
    });
}

// The reference's Count / Retrieve guards (static_multimap.h:258-270 CheckCount
// with detail/static_multimap/storage.h:29-35 Bytes; static_multiset.h CountImpl):
// the query array's byte size and n * Size() must be representable.
int count_guard(uint64_t n, uint64_t size, uint32_t key_bytes)
{
    if (n > ~0ull / key_bytes) return fail(B2CO_EOVERFLOW, "buffer byte size overflow");
    if (size && n > ~0ull / size) return fail(B2CO_EOVERFLOW, "potential total count overflow");
    return B2CO_OK;
}

}  // namespace

extern "C" {

// ---- StaticMultiset ---------------------------------------------------------------

int b2co_mset_create(uint64_t capacity, uint32_t key_bytes, uint64_t empty_key_bits, b2co_stream stream,
                     b2co_mset** out)
{
    if (!out) return fail(B2CO_EINVAL, "null output");
    *out = nullptr;
    if (capacity == 0) return fail(B2CO_EINVAL, "StaticMultiset: capacity must be positive");
    if (capacity > kMaxElements) return fail(B2CO_EINVAL, "StaticMultiset: capacity above 2^31");
    if (key_bytes != 4 && key_bytes != 8) return fail(B2CO_EINVAL, "StaticMultiset: keys are 4 or 8 bytes");
    auto* s = new (std::nothrow) b2co_mset;
    if (!s) return fail(B2CO_ENOMEM, "host allocation failed");
    s->capacity = capacity;
    s->kb = key_bytes;
    s->empty = mask_bits(empty_key_bits, key_bytes);
    s->tsize = table_size_for(capacity);
    cudaError_t e = cudaMalloc(&s->ordered, capacity * key_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&s->tkeys, s->tsize * key_bytes);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s->tcounts), s->tsize * 4);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&s->h_word), sizeof(uint64_t));
    if (e != cudaSuccess) {
        b2co_mset_destroy(s);
        return e == cudaErrorMemoryAllocation ? fail(B2CO_ENOMEM, "StaticMultiset allocation") : cuda_fail(e, "StaticMultiset");
    }
    if (int st = b2co_mset_clear(s, stream)) {
        b2co_mset_destroy(s);
        return st;
    }
    *out = s;
    return B2CO_OK;
}

int b2co_mset_destroy(b2co_mset* s)
{
    if (!s) return B2CO_OK;
    cudaFree(s->ordered);
    cudaFree(s->tkeys);
    cudaFree(s->tcounts);
    if (s->h_word) cudaFreeHost(s->h_word);
    s->scratch.release();
    delete s;
    return B2CO_OK;
}

int b2co_mset_capacity(b2co_mset const* s, uint64_t* c)
{
    if (int e = check_mset(s)) return e;
    if (!c) return fail(B2CO_EINVAL, "null output");
    *c = s->capacity;
    return B2CO_OK;
}

int b2co_mset_size(b2co_mset const* s, uint64_t* n)
{
    if (int e = check_mset(s)) return e;
    if (!n) return fail(B2CO_EINVAL, "null output");
    *n = s->size;
    return B2CO_OK;
}

int b2co_mset_clear(b2co_mset* s, b2co_stream st)
{
    if (int e = check_mset(s)) return e;
    return by_kb(s->kb, [&](auto k) { return mset_clear<decltype(k)::value>(s, cs(st)); });
}

static int mset_insert_any(b2co_mset* s, void const* keys, uint8_t const* stencil, bool use_stencil, uint64_t n,
                           b2co_stream st, uint64_t* failed)
{
    if (int e = check_mset(s)) return e;
    if (failed) *failed = 0;
    if (n == 0) return B2CO_OK;
    if (use_stencil && !stencil) return fail(B2CO_EINVAL, "StaticMultiset::InsertIf: null stencil");
    if (!keys) {  // static_multiset.h:161: a null key array reports every key failed
        if (failed) *failed = n;
        return B2CO_OK;
    }
    if (int e = check_batch(n)) return e;
    return by_kb(s->kb, [&](auto k) { return mset_insert<decltype(k)::value>(s, keys, stencil, n, cs(st), failed); });
}

int b2co_mset_insert(b2co_mset* s, void const* keys, uint64_t n, b2co_stream st, uint64_t* failed)
{
    return mset_insert_any(s, keys, nullptr, false, n, st, failed);
}

int b2co_mset_insert_if(b2co_mset* s, void const* keys, uint8_t const* stencil, uint64_t n, b2co_stream st,
                        uint64_t* failed)
{
    return mset_insert_any(s, keys, stencil, true, n, st, failed);
}

int b2co_mset_contains(b2co_mset* s, void const* keys, uint8_t* out, uint64_t n, b2co_stream st)
{
    return mset_query_any(s, keys, nullptr, false, out, n, st, 0);
}
int b2co_mset_contains_if(b2co_mset* s, void const* keys, uint8_t const* stencil, uint8_t* out, uint64_t n,
                          b2co_stream st)
{
    return mset_query_any(s, keys, stencil, true, out, n, st, 0);
}
int b2co_mset_find(b2co_mset* s, void const* keys, void* out, uint64_t n, b2co_stream st)
{
    return mset_query_any(s, keys, nullptr, false, out, n, st, 1);
}
int b2co_mset_find_if(b2co_mset* s, void const* keys, uint8_t const* stencil, void* out, uint64_t n, b2co_stream st)
{
    return mset_query_any(s, keys, stencil, true, out, n, st, 1);
}
int b2co_mset_count_each(b2co_mset* s, void const* keys, uint64_t* out, uint64_t n, b2co_stream st)
{
    return mset_query_any(s, keys, nullptr, false, out, n, st, 2);
}
int b2co_mset_count_each_outer(b2co_mset* s, void const* keys, uint64_t* out, uint64_t n, b2co_stream st)
{
    return mset_query_any(s, keys, nullptr, false, out, n, st, 3);
}

int b2co_mset_count(b2co_mset* s, void const* keys, uint64_t n, b2co_stream st, uint64_t* total)
{
    if (int e = check_mset(s)) return e;
    if (!total) return fail(B2CO_EINVAL, "null output");
    *total = 0;
    if (n == 0) return B2CO_OK;
    if (!keys) return fail(B2CO_EINVAL, "StaticMultiset: null nonempty buffer");
    if (int e = count_guard(n, s->size, s->kb)) return e;
    if (int e = check_batch(n)) return e;
    return by_kb(s->kb, [&](auto k) {
        return mset_count<decltype(k)::value>(s, keys, n, cs(st), total, false, nullptr, nullptr, 0);
    });
}

int b2co_mset_retrieve(b2co_mset* s, void const* keys, uint64_t n, void* probe_out, void* match_out,
                       uint64_t cap, b2co_stream st, uint64_t* written)
{
    if (int e = check_mset(s)) return e;
    if (!written) return fail(B2CO_EINVAL, "null output");
    *written = 0;
    if (n == 0) return B2CO_OK;
    if (!keys) return fail(B2CO_EINVAL, "StaticMultiset: null nonempty buffer");
    if (int e = count_guard(n, s->size, s->kb)) return e;
    if (int e = check_batch(n)) return e;
    uint64_t total = 0;
    int r = by_kb(s->kb, [&](auto k) {
        return mset_count<decltype(k)::value>(s, keys, n, cs(st), &total, true, probe_out, match_out, cap);
    });
    if (!r) *written = total;
    return r;
}

int b2co_mset_retrieve_all(b2co_mset* s, void* out, uint64_t cap, b2co_stream st, uint64_t* written)
{
    if (int e = check_mset(s)) return e;
    if (!written) return fail(B2CO_EINVAL, "null output");
    *written = 0;
    if (s->size > cap) return fail(B2CO_ERANGE, "StaticMultiset: output capacity too small");
    if (!s->size) return B2CO_OK;
    if (!out) return fail(B2CO_EINVAL, "StaticMultiset: null nonempty buffer");
    B2CO_CUDA(cudaMemcpyAsync(out, s->ordered, s->size * s->kb, cudaMemcpyDeviceToDevice, cs(st)));
    B2CO_CUDA(cudaStreamSynchronize(cs(st)));
    *written = s->size;
    return B2CO_OK;
}

// ---- StaticMultimap ---------------------------------------------------------------

int b2co_mmap_create(uint64_t capacity, uint32_t key_bytes, uint32_t value_bytes, uint64_t ek, uint64_t ev,
                     b2co_stream stream, b2co_mmap** out)
{
    if (!out) return fail(B2CO_EINVAL, "null output");
    *out = nullptr;
    if (capacity == 0) return fail(B2CO_EINVAL, "StaticMultimap: capacity must be positive");
    if (capacity > kMaxElements) return fail(B2CO_EINVAL, "StaticMultimap: capacity above 2^31");
    if ((key_bytes != 4 && key_bytes != 8) || (value_bytes != 4 && value_bytes != 8))
        return fail(B2CO_EINVAL, "StaticMultimap: keys and values are 4 or 8 bytes");
    auto* m = new (std::nothrow) b2co_mmap;
    if (!m) return fail(B2CO_ENOMEM, "host allocation failed");
    m->capacity = capacity;
    m->kb = key_bytes;
    m->vb = value_bytes;
    m->ek = mask_bits(ek, key_bytes);
    m->ev = mask_bits(ev, value_bytes);
    cudaError_t e = cudaMalloc(&m->dense, capacity * m->slot_bytes());
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&m->d_status), sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&m->h_word), sizeof(uint64_t));
    if (e != cudaSuccess) {
        b2co_mmap_destroy(m);
        return e == cudaErrorMemoryAllocation ? fail(B2CO_ENOMEM, "StaticMultimap allocation") : cuda_fail(e, "StaticMultimap");
    }
    if (int st = b2co_mmap_clear(m, stream)) {
        b2co_mmap_destroy(m);
        return st;
    }
    *out = m;
    return B2CO_OK;
}

int b2co_mmap_destroy(b2co_mmap* m)
{
    if (!m) return B2CO_OK;
    cudaFree(m->dense);
    cudaFree(m->tkeys);
    cudaFree(m->tcounts);
    cudaFree(m->toffsets);
    cudaFree(m->rec[0]);
    cudaFree(m->rec[1]);
    cudaFree(m->csr);
    cudaFree(m->d_status);
    if (m->h_word) cudaFreeHost(m->h_word);
    m->scratch.release();
    m->hist.release();
    delete m;
    return B2CO_OK;
}

int b2co_mmap_capacity(b2co_mmap const* m, uint64_t* c)
{
    if (int e = check_mmap(m)) return e;
    if (!c) return fail(B2CO_EINVAL, "null output");
    *c = m->capacity;
    return B2CO_OK;
}

int b2co_mmap_size(b2co_mmap const* m, uint64_t* n)
{
    if (int e = check_mmap(m)) return e;
    if (!n) return fail(B2CO_EINVAL, "null output");
    *n = m->size;
    return B2CO_OK;
}

int b2co_mmap_clear(b2co_mmap* m, b2co_stream)
{
    if (int e = check_mmap(m)) return e;
    m->size = 0;
    m->dirty = true;  // the next query builds an empty index
    return B2CO_OK;
}

static int mmap_insert_any(b2co_mmap* m, void const* pairs, uint8_t const* stencil, bool use_stencil, uint64_t n,
                           b2co_stream st, uint64_t* failed)
{
    if (int e = check_mmap(m)) return e;
    if (failed) *failed = 0;
    if (n == 0) return B2CO_OK;
    if (!pairs) return fail(B2CO_EINVAL, "StaticMultimap: null nonempty buffer");
    if (use_stencil && !stencil) return fail(B2CO_EINVAL, "StaticMultimap: null nonempty buffer");
    if (int e = check_batch(n)) return e;
    return by_kv(m->kb, m->vb, [&](auto k, auto v) {
        return mmap_insert<decltype(k)::value, decltype(v)::value>(m, pairs, stencil, n, cs(st), failed);
    });
}

int b2co_mmap_insert(b2co_mmap* m, void const* pairs, uint64_t n, b2co_stream st, uint64_t* failed)
{
    return mmap_insert_any(m, pairs, nullptr, false, n, st, failed);
}

int b2co_mmap_insert_if(b2co_mmap* m, void const* pairs, uint8_t const* stencil, uint64_t n, b2co_stream st,
                        uint64_t* failed)
{
    return mmap_insert_any(m, pairs, stencil, true, n, st, failed);
}

int b2co_mmap_contains(b2co_mmap* m, void const* keys, uint8_t* out, uint64_t n, b2co_stream st)
{
    return mmap_query_any(m, keys, nullptr, false, out, n, st, 0);
}
int b2co_mmap_contains_if(b2co_mmap* m, void const* keys, uint8_t const* stencil, uint8_t* out, uint64_t n,
                          b2co_stream st)
{
    return mmap_query_any(m, keys, stencil, true, out, n, st, 0);
}
int b2co_mmap_find(b2co_mmap* m, void const* keys, void* out, uint64_t n, b2co_stream st)
{
    return mmap_query_any(m, keys, nullptr, false, out, n, st, 1);
}
int b2co_mmap_find_if(b2co_mmap* m, void const* keys, uint8_t const* stencil, void* out, uint64_t n, b2co_stream st)
{
    return mmap_query_any(m, keys, stencil, true, out, n, st, 1);
}

static int mmap_count_any(b2co_mmap* m, void const* keys, uint64_t n, b2co_stream st, uint64_t* total, bool retrieve,
                          void* key_out, void* value_out, uint64_t cap)
{
    if (int e = check_mmap(m)) return e;
    *total = 0;
    if (n == 0) return B2CO_OK;
    if (!keys) return fail(B2CO_EINVAL, "StaticMultimap: null nonempty buffer");
    if (int e = count_guard(n, m->size, m->kb)) return e;
    if (int e = check_batch(n)) return e;
    return by_kv(m->kb, m->vb, [&](auto k, auto v) -> int {
        constexpr int KB = decltype(k)::value, VB = decltype(v)::value;
        cudaStream_t s = cs(st);
        if (int e = mmap_build<KB, VB>(m, s)) return e;
        if (int e = m->scratch.reserve(scan_scratch_words(n) * 8)) return e;
        uint64_t* sc = m->scratch.as<uint64_t>();
        MmapCount<KB> f{m->table<KB>(), static_cast<KeyWord<KB> const*>(keys)};
        if (int e = tile_scan(f, NoAct{}, n, sc, false, s)) return e;
        if (int e = read_word(sc + (n + kTile - 1) / kTile, m->h_word, s, total)) return e;
        if (!retrieve || *total == 0) return B2CO_OK;
        if (*total > cap) return fail(B2CO_ERANGE, "StaticMultimap: output capacity is insufficient");
        if (!key_out || !value_out) return fail(B2CO_EINVAL, "StaticMultimap: null nonempty buffer");
        MmapRetrieve<KB, VB> act{m->table<KB>(), static_cast<KeyWord<KB> const*>(keys), m->csr,
                                 static_cast<KeyWord<KB>*>(key_out), value_out};
        if (int e = apply_scanned(f, act, n, sc, s)) return e;
        B2CO_CUDA(cudaStreamSynchronize(s));
        return B2CO_OK;
    });
}

int b2co_mmap_count(b2co_mmap* m, void const* keys, uint64_t n, b2co_stream st, uint64_t* total)
{
    if (!total) return fail(B2CO_EINVAL, "null output");
    return mmap_count_any(m, keys, n, st, total, false, nullptr, nullptr, 0);
}

int b2co_mmap_retrieve(b2co_mmap* m, void const* keys, uint64_t n, void* key_out, void* value_out, uint64_t cap,
                       b2co_stream st, uint64_t* written)
{
    if (!written) return fail(B2CO_EINVAL, "null output");
    uint64_t total = 0;
    *written = 0;
    int r = mmap_count_any(m, keys, n, st, &total, true, key_out, value_out, cap);
    if (!r) *written = total;
    return r;
}

int b2co_mmap_retrieve_all(b2co_mmap* m, void* key_out, void* value_out, uint64_t cap, b2co_stream st,
                           uint64_t* written)
{
    if (int e = check_mmap(m)) return e;
    if (!written) return fail(B2CO_EINVAL, "null output");
    *written = 0;
    if (m->size > cap) return fail(B2CO_ERANGE, "StaticMultimap: output capacity is insufficient");
    if (!m->size) return B2CO_OK;
    if (!key_out || !value_out) return fail(B2CO_EINVAL, "StaticMultimap: null nonempty buffer");
    int r = by_kv(m->kb, m->vb, [&](auto k, auto v) -> int {
        constexpr int KB = decltype(k)::value, VB = decltype(v)::value;
        using Raw = typename SlotT<KB, VB>::Raw;
        k_mmap_export<KB, VB><<<blocks_for(m->size), 256, 0, cs(st)>>>(static_cast<Raw const*>(m->dense), m->size,
                                                                        static_cast<KeyWord<KB>*>(key_out), value_out);
        B2CO_CUDA(cudaGetLastError());
        B2CO_CUDA(cudaStreamSynchronize(cs(st)));
        return B2CO_OK;
    });
    if (!r) *written = m->size;
    return r;
}

}  // extern "C"
