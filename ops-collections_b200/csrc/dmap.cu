// dmap.cu -- DynamicMap<K,T>: a growing list of StaticMap submaps
// (include/dynamic_map.h, detail/dynamic_map/kernels.h).
//
// Same orchestration as the reference: inserts go to the active (last)
// submap; a new submap is added when the active one runs out of room (max
// load 0.6, minimum 10,000 spare, x2 growth), and may be prepared (cleared)
// ahead of time on a side stream; lookups fan out over the non-empty submaps
// and merge on the device; inserts into a grown map skip keys already present
// in an older submap (exact dedup) unless the caller promises unique keys.
#include <cmath>
#include <memory>
#include <new>
#include <vector>

#include "b2co_host.h"
#include "oa_kernels.cuh"

using namespace b2co;

int b2co_oa_create_ex(b2co_oa_desc const* d, uint64_t requested, bool clear, b2co_stream stream, b2co_oa_table** out);

namespace {

cudaStream_t cs(b2co_stream s) { return reinterpret_cast<cudaStream_t>(s); }
b2co_stream bs(cudaStream_t s) { return reinterpret_cast<b2co_stream>(s); }

// MergeFind (detail/dynamic_map/kernels.h:73-96): take the submap's answer
// where the running answer is still the empty payload (a key lives in at most
// one submap).
template <class W>
__global__ void __launch_bounds__(256) k_merge_find(W* out, W const* tmp, W empty, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (out[i] == empty) out[i] = tmp[i];
}

// MergeContains (kernels.h:98-112): bitwise OR of the 1-byte flags.
__global__ void __launch_bounds__(256) k_merge_contains(uint8_t* out, uint8_t const* tmp, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (tmp[i]) out[i] = 1;
}

// ExtractKeys (kernels.h:34-48): the keys of a pair array.
template <class S>
__global__ void __launch_bounds__(256) k_extract_keys(void* keys, void const* pairs, uint32_t n)
{
    using K = WordT<S::key_bytes>;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        reinterpret_cast<K*>(keys)[i] = K(S::key(Io<S>::load_pair(pairs, i)));
}

// notmask[i] = !mask[i]; counter += number of zero flags (CountZero, kernels.h:50-70).
__global__ void __launch_bounds__(256) k_invert_count(uint8_t const* mask, uint8_t* notmask, uint32_t n,
                                                      unsigned long long* counter)
{
    uint32_t zeros = 0;
    uint32_t const stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        uint32_t i = base + (threadIdx.x & 31);
        if (i < n) {
            uint8_t z = mask[i] == 0;
            notmask[i] = z;
            zeros += z;
        }
    }
    warp_add_counter(counter, zeros);
}

struct TableDel {
    void operator()(b2co_oa_table* t) const { b2co_oa_destroy(t); }
};
using TablePtr = std::unique_ptr<b2co_oa_table, TableDel>;

}  // namespace

struct b2co_dmap {
    static constexpr uint64_t kMinInsert = 10000;
    static constexpr double kMaxLoad = 0.60f;  // the reference stores it as a float
    static constexpr uint64_t kGrowth = 2;
    static constexpr uint64_t kSubBatch = 800000;

    b2co_oa_desc desc{};
    std::vector<TablePtr> submaps;
    std::vector<uint64_t> sizes;
    uint64_t size = 0, total_capacity = 0, next_capacity = 0;
    // device scratch, grown on demand
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    void* dedup = nullptr;  // keys | mask | notmask
    size_t dedup_bytes = 0, keys_bytes = 0, mask_bytes = 0;
    unsigned long long* d_counter = nullptr;
    unsigned long long* h_counter = nullptr;
    // background preparation of the next submap
    TablePtr next;
    uint64_t next_cap = 0;
    cudaStream_t prep = nullptr;
    cudaEvent_t prep_ev = nullptr;

    ~b2co_dmap()
    {
        if (next && prep) cudaStreamSynchronize(prep);
        next.reset();
        submaps.clear();
        if (scratch) cudaFree(scratch);
        if (dedup) cudaFree(dedup);
        if (d_counter) cudaFree(d_counter);
        if (h_counter) cudaFreeHost(h_counter);
        if (prep_ev) cudaEventDestroy(prep_ev);
        if (prep) cudaStreamDestroy(prep);
    }

    uint32_t pair_bytes() const
    {
        uint32_t const raw = desc.key_bytes + desc.value_bytes;
        return raw <= 4 ? 4 : (raw <= 8 ? 8 : 16);
    }
    uint64_t capacity_of(size_t i) const
    {
        uint64_t c = 0;
        b2co_oa_capacity(submaps[i].get(), &c);
        return c;
    }
    uint64_t usable(uint64_t cap) const
    {
        uint64_t u = uint64_t(std::floor(double(float(kMaxLoad)) * double(cap)));
        return u > kMinInsert ? u - kMinInsert : 0;
    }
    size_t active() const { return submaps.size() - 1; }
    uint64_t active_room() const
    {
        uint64_t u = usable(capacity_of(active()));
        return u > sizes[active()] ? u - sizes[active()] : 0;
    }
    size_t first_nonempty() const
    {
        for (size_t s = 0; s < submaps.size(); ++s)
            if (sizes[s]) return s;
        return submaps.size();
    }
    bool nonempty_before(size_t a) const
    {
        for (size_t s = 0; s < a; ++s)
            if (sizes[s]) return true;
        return false;
    }
    bool nonempty_after(size_t b) const
    {
        for (size_t s = b + 1; s < submaps.size(); ++s)
            if (sizes[s]) return true;
        return false;
    }
    uint64_t grow_target(uint64_t min_usable) const
    {
        uint64_t g = size * kGrowth;
        return g > min_usable ? g : min_usable;
    }

    int add_submap(uint64_t requested, bool clear, cudaStream_t s, TablePtr& out)
    {
        b2co_oa_table* t = nullptr;
        if (int st = b2co_oa_create_ex(&desc, requested, clear, bs(s), &t)) return st;
        out.reset(t);
        return B2CO_OK;
    }

    int push(TablePtr t)
    {
        submaps.push_back(std::move(t));
        sizes.push_back(0);
        total_capacity += capacity_of(active());
        return B2CO_OK;
    }

    int discard_prepared()
    {
        if (next) {
            B2CO_CUDA(cudaStreamSynchronize(prep));
            next.reset();
        }
        next_cap = 0;
        return B2CO_OK;
    }

    // StartPrepareNext (dynamic_map.h:463-482): create the next submap and clear it on the side stream.
    int start_prepare(uint64_t min_usable)
    {
        if (next || !prep) return B2CO_OK;
        uint64_t cap = next_capacity;
        while (usable(cap) < grow_target(min_usable)) cap *= kGrowth;
        if (int st = add_submap(cap, false, prep, next)) return st;
        if (int st = b2co_oa_clear_async(next.get(), bs(prep))) return st;
        cudaError_t e = cudaEventRecord(prep_ev, prep);
        if (e != cudaSuccess) {
            discard_prepared();
            return cuda_fail(e, "DynamicMap::StartPrepareNext::cudaEventRecord");
        }
        next_cap = cap;
        return B2CO_OK;
    }

    // ActivateNext (dynamic_map.h:485-507).
    int activate_next(uint64_t min_usable, cudaStream_t s)
    {
        if (next && usable(next_cap) >= min_usable) {
            B2CO_CUDA(cudaStreamWaitEvent(s, prep_ev, 0));
            push(std::move(next));
            next_capacity = next_cap * kGrowth;
            next_cap = 0;
            return B2CO_OK;
        }
        if (int st = discard_prepared()) return st;
        uint64_t cap = next_capacity;
        while (usable(cap) < min_usable) cap *= kGrowth;
        TablePtr t;
        if (int st = add_submap(cap, true, s, t)) return st;
        push(std::move(t));
        next_capacity = cap * kGrowth;
        return B2CO_OK;
    }

    int ensure_active_room(uint64_t n, cudaStream_t s)
    {
        if (active_room() >= n) return B2CO_OK;
        return activate_next(grow_target(n), s);
    }

    int ensure_scratch(size_t bytes)
    {
        if (scratch_bytes >= bytes && scratch) return B2CO_OK;
        if (scratch) cudaFree(scratch);
        scratch = nullptr;
        scratch_bytes = 0;
        B2CO_CUDA(cudaMalloc(&scratch, bytes));
        scratch_bytes = bytes;
        return B2CO_OK;
    }

    int ensure_dedup(uint64_t n)
    {
        size_t kb = ((n * desc.key_bytes + 63) / 64) * 64;
        size_t mb = ((n + 63) / 64) * 64;
        size_t bytes = kb + 2 * mb;
        keys_bytes = kb;
        mask_bytes = mb;
        if (dedup_bytes >= bytes && dedup) return B2CO_OK;
        if (dedup) cudaFree(dedup);
        dedup = nullptr;
        dedup_bytes = 0;
        B2CO_CUDA(cudaMalloc(&dedup, bytes));
        dedup_bytes = bytes;
        return B2CO_OK;
    }
    uint8_t* d_keys() const { return static_cast<uint8_t*>(dedup); }
    uint8_t* d_mask() const { return d_keys() + keys_bytes; }
    uint8_t* d_notmask() const { return d_mask() + mask_bytes; }

    template <class S>
    static void launch_extract(void* keys, void const* pairs, uint32_t n, cudaStream_t s)
    {
        auto k = k_extract_keys<S>;
        k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(keys, pairs, n);
    }

    int extract_keys(void const* pairs, uint32_t n, cudaStream_t s)
    {
        uint32_t kb = desc.key_bytes, vb = desc.value_bytes;  // the key's bits, whatever its kind
        if (kb == 2) launch_extract<SlotT<2, 2>>(d_keys(), pairs, n, s);
        else if (kb == 4 && vb == 4) launch_extract<SlotT<4, 4>>(d_keys(), pairs, n, s);
        else if (kb == 4 && vb == 8) launch_extract<SlotT<4, 8>>(d_keys(), pairs, n, s);
        else if (kb == 8 && vb == 4) launch_extract<SlotT<8, 4>>(d_keys(), pairs, n, s);
        else launch_extract<SlotT<8, 8>>(d_keys(), pairs, n, s);
        B2CO_CUDA(cudaGetLastError());
        return B2CO_OK;
    }

    // BuildContainsMask (dynamic_map.h:414-432) plus the inverted mask and its
    // zero count; mask[i] = key i lives in an older non-empty submap.
    int build_masks(void const* pairs, uint64_t n, cudaStream_t s, uint64_t* candidates)
    {
        if (int st = ensure_dedup(n)) return st;
        if (int st = extract_keys(pairs, uint32_t(n), s)) return st;
        bool first = true;
        for (size_t i = 0; i < active(); ++i) {
            if (!sizes[i]) continue;
            if (first) {
                if (int st = b2co_oa_contains_async(submaps[i].get(), d_keys(), d_mask(), n, bs(s))) return st;
                first = false;
            } else {
                if (int st = b2co_oa_contains_async(submaps[i].get(), d_keys(), d_notmask(), n, bs(s))) return st;
                k_merge_contains<<<grid_for((void const*)k_merge_contains, 256, n, 256), 256, 0, s>>>(
                    d_mask(), d_notmask(), uint32_t(n));
                B2CO_CUDA(cudaGetLastError());
            }
        }
        B2CO_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), s));
        k_invert_count<<<grid_for((void const*)k_invert_count, 256, n, 256), 256, 0, s>>>(d_mask(), d_notmask(),
                                                                                           uint32_t(n), d_counter);
        B2CO_CUDA(cudaGetLastError());
        B2CO_CUDA(cudaMemcpyAsync(h_counter, d_counter, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        B2CO_CUDA(cudaStreamSynchronize(s));
        *candidates = *h_counter;
        return B2CO_OK;
    }

    // InsertChunk (dynamic_map.h:523-545).
    int insert_chunk(void const* pairs, uint64_t n, cudaStream_t s, uint64_t* inserted)
    {
        size_t a = active();
        uint64_t ins = 0;
        if (!nonempty_before(a)) {
            uint64_t failed = 0;
            if (int st = b2co_oa_insert(submaps[a].get(), pairs, n, bs(s), &failed)) return st;
            ins = n - failed;
        } else {
            uint64_t candidates = 0, failed = 0;
            if (int st = build_masks(pairs, n, s, &candidates)) return st;
            if (int st = b2co_oa_insert_if(submaps[a].get(), pairs, d_notmask(), n, bs(s), &failed)) return st;
            ins = candidates - failed;
        }
        sizes[a] += ins;
        size += ins;
        *inserted = ins;
        return B2CO_OK;
    }

    // InsertOrAssignChunk (dynamic_map.h:549-575): only new keys are counted.
    int insert_or_assign_chunk(void const* pairs, uint64_t n, cudaStream_t s, uint64_t* inserted)
    {
        size_t a = active();
        uint64_t ins = 0;
        if (!nonempty_before(a)) {
            uint64_t failed = 0, assigned = 0;
            if (int st = b2co_oa_insert_or_assign(submaps[a].get(), pairs, n, bs(s), &failed, &assigned)) return st;
            ins = n - failed - assigned;
        } else {
            uint64_t candidates = 0, failed = 0;
            if (int st = build_masks(pairs, n, s, &candidates)) return st;
            for (size_t i = 0; i < a; ++i) {
                if (!sizes[i]) continue;
                if (int st = b2co_oa_assign_if_async(submaps[i].get(), pairs, d_mask(), n, bs(s))) return st;
            }
            if (int st = b2co_oa_assign_if_async(submaps[a].get(), pairs, d_notmask(), n, bs(s))) return st;
            if (int st = b2co_oa_insert_if(submaps[a].get(), pairs, d_notmask(), n, bs(s), &failed)) return st;
            ins = candidates - failed;
        }
        sizes[a] += ins;
        size += ins;
        *inserted = ins;
        return B2CO_OK;
    }
};

int b2co_dmap_check(b2co_dmap const* m)
{
    if (!m || m->submaps.empty()) return fail(B2CO_ELOGIC, "DynamicMap is null or moved-from");
    return B2CO_OK;
}

template <class W>
static int merge_find(void* out, void const* tmp, uint64_t empty, uint64_t n, cudaStream_t s)
{
    auto k = k_merge_find<W>;
    k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(static_cast<W*>(out), static_cast<W const*>(tmp), W(empty),
                                                           uint32_t(n));
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

extern "C" {

int b2co_dmap_create(b2co_oa_desc const* d, uint64_t initial_capacity, b2co_stream stream, b2co_dmap** out)
{
    if (!d || !out) return fail(B2CO_EINVAL, "null descriptor or output");
    *out = nullptr;
    if (d->value_bytes == 0) return fail(B2CO_EINVAL, "DynamicMap needs a payload (value_bytes > 0)");
    // the submaps check the layout and the key kind (2-byte keys with 2-byte
    // payloads; 4- and 8-byte keys with 4- or 8-byte payloads; integer or float)
    uint64_t kmask = d->key_bytes >= 8 ? ~0ull : ((1ull << (8 * d->key_bytes)) - 1);
    if ((d->empty_key_bits & kmask) == (d->erased_key_bits & kmask))
        return fail(B2CO_EINVAL, "DynamicMap: emptyKey and erasedKey must differ");
    auto* m = new (std::nothrow) b2co_dmap;
    if (!m) return fail(B2CO_ENOMEM, "host allocation failed");
    std::unique_ptr<b2co_dmap> guard(m);
    m->desc = *d;
    TablePtr t;
    if (int st = m->add_submap(initial_capacity, true, cs(stream), t)) return st;
    m->push(std::move(t));
    m->next_capacity = m->capacity_of(0) * b2co_dmap::kGrowth;
    B2CO_CUDA(cudaMalloc(&m->d_counter, sizeof(unsigned long long)));
    B2CO_CUDA(cudaMallocHost(&m->h_counter, sizeof(unsigned long long)));
    // a failed side stream is not fatal: growth then happens synchronously
    if (cudaStreamCreateWithFlags(&m->prep, cudaStreamNonBlocking) == cudaSuccess) {
        if (cudaEventCreateWithFlags(&m->prep_ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaStreamDestroy(m->prep);
            m->prep = nullptr;
        }
    } else {
        m->prep = nullptr;
    }
    *out = guard.release();
    return B2CO_OK;
}

int b2co_dmap_destroy(b2co_dmap* m)
{
    delete m;
    return B2CO_OK;
}

int b2co_dmap_size(b2co_dmap const* m, uint64_t* v)
{
    if (int st = b2co_dmap_check(m)) return st;
    *v = m->size;
    return B2CO_OK;
}

int b2co_dmap_capacity(b2co_dmap const* m, uint64_t* v)
{
    if (int st = b2co_dmap_check(m)) return st;
    *v = m->total_capacity;
    return B2CO_OK;
}

int b2co_dmap_num_submaps(b2co_dmap const* m, uint64_t* v)
{
    if (int st = b2co_dmap_check(m)) return st;
    *v = m->submaps.size();
    return B2CO_OK;
}

// Reserve (dynamic_map.h:142-166).
int b2co_dmap_reserve(b2co_dmap* m, uint64_t n, b2co_stream s)
{
    if (int st = b2co_dmap_check(m)) return st;
    uint64_t remaining = n;
    size_t idx = 0;
    while (remaining > 0) {
        uint64_t cap;
        if (idx < m->submaps.size()) {
            cap = m->capacity_of(idx);
        } else {
            cap = m->next_capacity;
            TablePtr t;
            if (int st = m->add_submap(cap, true, cs(s), t)) return st;
            m->push(std::move(t));
            m->next_capacity = cap * b2co_dmap::kGrowth;
        }
        uint64_t u = m->usable(cap);
        if (u >= remaining) break;
        remaining -= u;
        ++idx;
    }
    return B2CO_OK;
}

// Insert (dynamic_map.h:168-219).
int b2co_dmap_insert(b2co_dmap* m, void const* pairs, uint64_t n, int mode, b2co_stream stream, uint64_t* inserted)
{
    uint64_t dummy;
    if (!inserted) inserted = &dummy;
    *inserted = 0;
    if (int st = b2co_dmap_check(m)) return st;
    if (n == 0 || !pairs) return B2CO_OK;
    cudaStream_t s = cs(stream);
    if (int st = m->ensure_active_room(n, s)) return st;
    size_t a = m->active();
    uint32_t const pb = m->pair_bytes();
    if (mode == 1) {  // kAppendUnique: optimistic count, no per-batch sync
        for (uint64_t off = 0; off < n; off += b2co_dmap::kSubBatch) {
            uint64_t cur = n - off < b2co_dmap::kSubBatch ? n - off : b2co_dmap::kSubBatch;
            if (int st = b2co_oa_insert_async(m->submaps[a].get(), static_cast<char const*>(pairs) + off * pb, cur,
                                              stream))
                return st;
        }
        m->sizes[a] += n;
        m->size += n;
        *inserted = n;
        return B2CO_OK;
    }
    if (mode != 0) return fail(B2CO_EINVAL, "unknown DynamicMap insert mode");
    if (!m->nonempty_before(a)) {
        uint64_t failed = 0;
        if (int st = b2co_oa_insert(m->submaps[a].get(), pairs, n, stream, &failed)) return st;
        uint64_t ins = n >= failed ? n - failed : 0;
        m->sizes[a] += ins;
        m->size += ins;
        *inserted = ins;
        return B2CO_OK;
    }
    uint64_t total = 0, off = 0;
    while (off < n) {
        uint64_t room = m->active_room();
        if (room == 0) {
            if (int st = m->activate_next(m->grow_target(n - off), s)) return st;
            continue;
        }
        if (room < (n - off) * 2)
            if (int st = m->start_prepare(n - off)) return st;
        uint64_t chunk = n - off < room ? n - off : room, ins = 0;
        if (int st = m->insert_chunk(static_cast<char const*>(pairs) + off * pb, chunk, s, &ins)) return st;
        total += ins;
        off += chunk;
    }
    *inserted = total;
    return B2CO_OK;
}

// InsertOrAssign (dynamic_map.h:237-260): returns the number of new keys.
int b2co_dmap_insert_or_assign(b2co_dmap* m, void const* pairs, uint64_t n, b2co_stream stream, uint64_t* done)
{
    uint64_t dummy;
    if (!done) done = &dummy;
    *done = 0;
    if (int st = b2co_dmap_check(m)) return st;
    if (n == 0 || !pairs) return B2CO_OK;
    cudaStream_t s = cs(stream);
    if (int st = m->ensure_active_room(n, s)) return st;
    uint32_t const pb = m->pair_bytes();
    uint64_t total = 0, off = 0;
    while (off < n) {
        uint64_t room = m->active_room();
        if (room == 0) {
            if (int st = m->activate_next(m->grow_target(n - off), s)) return st;
            continue;
        }
        if (room < (n - off) * 2)
            if (int st = m->start_prepare(n - off)) return st;
        uint64_t chunk = n - off < room ? n - off : room, ins = 0;
        if (int st = m->insert_or_assign_chunk(static_cast<char const*>(pairs) + off * pb, chunk, s, &ins)) return st;
        total += ins;
        off += chunk;
    }
    *done = total;
    return B2CO_OK;
}

// Find (dynamic_map.h:262-290).
int b2co_dmap_find(b2co_dmap* m, void const* keys, void* out, uint64_t n, b2co_stream stream)
{
    if (int st = b2co_dmap_check(m)) return st;
    if (n == 0 || !keys || !out) return B2CO_OK;
    cudaStream_t s = cs(stream);
    size_t base = m->first_nonempty();
    if (base == m->submaps.size()) return b2co_oa_find(m->submaps[0].get(), keys, out, n, stream);
    if (int st = b2co_oa_find_async(m->submaps[base].get(), keys, out, n, stream)) return st;
    if (m->nonempty_after(base)) {
        uint32_t vb = m->desc.value_bytes;
        if (int st = m->ensure_scratch(n * vb)) return st;
        for (size_t i = base + 1; i < m->submaps.size(); ++i) {
            if (!m->sizes[i]) continue;
            if (int st = b2co_oa_find_async(m->submaps[i].get(), keys, m->scratch, n, stream)) return st;
            int st = vb == 8   ? merge_find<unsigned long long>(out, m->scratch, m->desc.empty_value_bits, n, s)
                     : vb == 4 ? merge_find<uint32_t>(out, m->scratch, m->desc.empty_value_bits, n, s)
                               : merge_find<unsigned short>(out, m->scratch, m->desc.empty_value_bits, n, s);
            if (st) return st;
        }
    }
    B2CO_CUDA(cudaStreamSynchronize(s));
    return B2CO_OK;
}

// Contains (dynamic_map.h:292-316).
int b2co_dmap_contains(b2co_dmap* m, void const* keys, uint8_t* out, uint64_t n, b2co_stream stream)
{
    if (int st = b2co_dmap_check(m)) return st;
    if (n == 0 || !keys || !out) return B2CO_OK;
    cudaStream_t s = cs(stream);
    size_t base = m->first_nonempty();
    if (base == m->submaps.size()) return b2co_oa_contains(m->submaps[0].get(), keys, out, n, stream);
    if (int st = b2co_oa_contains_async(m->submaps[base].get(), keys, out, n, stream)) return st;
    if (m->nonempty_after(base)) {
        if (int st = m->ensure_scratch(n)) return st;
        for (size_t i = base + 1; i < m->submaps.size(); ++i) {
            if (!m->sizes[i]) continue;
            uint8_t* tmp = static_cast<uint8_t*>(m->scratch);
            if (int st = b2co_oa_contains_async(m->submaps[i].get(), keys, tmp, n, stream)) return st;
            k_merge_contains<<<grid_for((void const*)k_merge_contains, 256, n, 256), 256, 0, s>>>(out, tmp,
                                                                                                   uint32_t(n));
            B2CO_CUDA(cudaGetLastError());
        }
    }
    B2CO_CUDA(cudaStreamSynchronize(s));
    return B2CO_OK;
}

// Erase (dynamic_map.h:318-335).
int b2co_dmap_erase(b2co_dmap* m, void const* keys, uint64_t n, b2co_stream stream, uint64_t* erased)
{
    uint64_t dummy;
    if (!erased) erased = &dummy;
    *erased = 0;
    if (int st = b2co_dmap_check(m)) return st;
    if (n == 0 || !keys) return B2CO_OK;
    uint64_t total = 0;
    for (size_t i = 0; i < m->submaps.size(); ++i) {
        if (!m->sizes[i]) continue;
        uint64_t failed = 0;
        if (int st = b2co_oa_erase(m->submaps[i].get(), keys, n, stream, &failed)) return st;
        uint64_t del = n - failed;
        m->sizes[i] -= m->sizes[i] >= del ? del : m->sizes[i];
        total += del;
    }
    m->size -= m->size >= total ? total : m->size;
    *erased = total;
    return B2CO_OK;
}

// Clear (dynamic_map.h:349-357).
int b2co_dmap_clear(b2co_dmap* m, b2co_stream stream)
{
    if (int st = b2co_dmap_check(m)) return st;
    if (int st = m->discard_prepared()) return st;
    for (auto& t : m->submaps)
        if (int st = b2co_oa_clear(t.get(), stream)) return st;
    for (auto& x : m->sizes) x = 0;
    m->size = 0;
    return B2CO_OK;
}

}  // extern "C"
