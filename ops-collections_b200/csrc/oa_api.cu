// oa_api.cu -- C ABI of the open-addressing containers (StaticMap/StaticSet).
//
// Host conventions follow detail/open_addressing/open_addressing_impl.h: zero
// items is a no-op, a NULL input makes a sync insert report every item failed
// and an async call return, batches beyond the kernel index range are a
// length error, sync calls synchronize the stream and read the counters back.
#include <cstring>
#include <new>

#include "b2co_host.h"
#include "oa_kernels.cuh"

using namespace b2co;

namespace b2co {

OaOps const* oa_ops_for(uint32_t kb, uint32_t vb, uint32_t kind)
{
    if (kind == B2CO_KEY_INTEGER) {
        if (kb == 2 && vb == 0) return &kOpsSet2;
        if (kb == 2 && vb == 2) return &kOpsMap22;
        if (kb == 4 && vb == 0) return &kOpsSet4;
        if (kb == 8 && vb == 0) return &kOpsSet8;
        if (kb == 4 && vb == 4) return &kOpsMap44;
        if (kb == 4 && vb == 8) return &kOpsMap48;
        if (kb == 8 && vb == 4) return &kOpsMap84;
        if (kb == 8 && vb == 8) return &kOpsMap88;
    } else if (kind == B2CO_KEY_FLOAT) {
        if (kb == 2 && vb == 0) return &kOpsSet2F;
        if (kb == 2 && vb == 2) return &kOpsMap22F;
        if (kb == 4 && vb == 0) return &kOpsSet4F;
        if (kb == 4 && vb == 4) return &kOpsMap44F;
        if (kb == 4 && vb == 8) return &kOpsMap48F;
        if (kb == 8 && vb == 0) return &kOpsSet8F;
        if (kb == 8 && vb == 4) return &kOpsMap84F;
        if (kb == 8 && vb == 8) return &kOpsMap88F;
    }
    return nullptr;
}

uint32_t oa_slot_bytes(uint32_t kb, uint32_t vb)
{
    if (vb == 0) return kb;
    uint32_t const sum = kb + vb, align = sum <= 4 ? 4 : (sum <= 8 ? 8 : 16);
    uint32_t const end = (kb + vb - 1) / vb * vb + vb;
    return (end + align - 1) / align * align;
}

}  // namespace b2co

// Staging slots (and pipeline streams) of the host-buffer Find.
constexpr int kHostSlots = 3;

struct b2co_oa_table {
    b2co_oa_desc desc{};
    OaArgs args{};
    OaOps const* ops = nullptr;
    uint64_t capacity = 0;
    int device = 0;
    unsigned long long* d_counters = nullptr;  // [failed, assigned]
    unsigned long long* h_counters = nullptr;  // pinned mirror
    // first-wins InsertAndFind scratch, grown on demand
    uint32_t* d_pos = nullptr;
    uint64_t pos_cap = 0;
    ScratchOrder first_wins_order;  // pos, the two bitmaps and owner[] serve one batch at a time
    uint32_t* d_newbits = nullptr;
    uint32_t* d_owner = nullptr;
    // host-buffer Find pipeline
    void* stage = nullptr;
    uint64_t stage_keys = 0;
    cudaStream_t pipe[kHostSlots] = {};
    cudaEvent_t ev[kHostSlots + 1] = {};  // per-stream completion, then the caller's start
    uint32_t find_lanes = 0, find_items = 0;
};

namespace {

uint64_t mask_bytes(uint64_t v, uint32_t n) { return n >= 8 ? v : (v & ((1ull << (8 * n)) - 1ull)); }

uint32_t slot_bytes(uint32_t kb, uint32_t vb) { return oa_slot_bytes(kb, vb); }

int check_table(b2co_oa_table const* t)
{
    if (!t || !t->args.slots) return fail(B2CO_ELOGIC, "table is null or has no storage");
    return B2CO_OK;
}

int check_batch(uint64_t n)
{
    if (n > kMaxBatch) return fail(B2CO_ERANGE, "OpenAddressing: batch size exceeds the kernel index range");
    return B2CO_OK;
}

cudaStream_t cs(b2co_stream s) { return reinterpret_cast<cudaStream_t>(s); }

// Default lookup shape per layout; b2co_oa_set_find_shape overrides it per table.
// Tables at most this large (about 2.5 times the 126 MB L2) are served mostly
// from L2, and the keys in flight per warp set their rate: measured on int64
// tables, two-lane lookups beat four-lane ones by 1.39x at 70 MB, 1.17x at 130 MB
// and 1.21x at 260 MB and lose by 8% at 520 MB; one-lane-per-key writes win by
// 1.7x at 70 and 130 MB and 1.45x at 260 MB and lose by 11% at 520 MB.
constexpr uint64_t kSmallTableBytes = uint64_t(320) << 20;

uint64_t table_bytes(b2co_oa_table const* t)
{
    return uint64_t(t->capacity) * slot_bytes(t->desc.key_bytes, t->desc.value_bytes);
}
bool small_table(b2co_oa_table const* t) { return table_bytes(t) <= kSmallTableBytes; }

// Writes to small tables run one lane per key (the reference's scan as
// written); larger tables take the cooperative default.
void default_write_shape(b2co_oa_table* t) { t->args.write_shape = small_table(t) ? (1u << 8) | 1u : 0u; }

void default_shape(b2co_oa_table* t)
{
    if (t->desc.bucket_size == 1) {
        t->find_lanes = 1;  // a one-slot window needs no cooperation
        t->find_items = 4;
    } else {
        // keys staged per warp, keys that probe on past their first window
        // queued and followed a pass at a time; four lanes per window (a 64-byte
        // row of 16-byte slots per load) with two windows in flight, or two
        // lanes and one window for 4-byte slots and for small tables (measured
        // best per layout and size, see kSmallTableBytes)
        uint32_t const sb = slot_bytes(t->desc.key_bytes, t->desc.value_bytes);
        bool const narrow = sb <= 4 || small_table(t);
        t->find_lanes = narrow ? 2 : 4;
        t->find_items = (narrow ? 1 : 2) | kShapeDeferred;
    }
}

unsigned int* status_word(b2co_oa_table* t) { return reinterpret_cast<unsigned int*>(t->d_counters + 2); }

int launch_find(b2co_oa_table* t, bool contains, void const* keys, uint8_t const* stencil, void* out, uint64_t n,
                cudaStream_t s)
{
    return t->ops->find(t->args, t->desc.bucket_size, t->find_lanes, t->find_items, contains, keys, stencil, out,
                        uint32_t(n), wait_ctl(status_word(t)), s);
}

// Reads (and clears) the table's device status word; a set word means a
// bounded device wait expired in some earlier kernel on this table.
int check_status(b2co_oa_table* t, cudaStream_t s)
{
    B2CO_CUDA(cudaMemcpyAsync(t->h_counters + 2, t->d_counters + 2, sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, s));
    B2CO_CUDA(cudaStreamSynchronize(s));
    if (t->h_counters[2] != 0) {
        B2CO_CUDA(cudaMemsetAsync(t->d_counters + 2, 0, sizeof(unsigned long long), s));
        B2CO_CUDA(cudaStreamSynchronize(s));
        return fail(B2CO_ETIMEOUT, "a bounded device wait expired (bulk key copy did not complete in time)");
    }
    return B2CO_OK;
}

int sync_counters(b2co_oa_table* t, cudaStream_t s, int words)
{
    B2CO_CUDA(cudaMemcpyAsync(t->h_counters, t->d_counters, sizeof(unsigned long long) * words,
                              cudaMemcpyDeviceToHost, s));
    B2CO_CUDA(cudaStreamSynchronize(s));
    return B2CO_OK;
}

int ensure_first_wins_scratch(b2co_oa_table* t, uint64_t n)
{
    if (!t->d_newbits) {
        uint64_t words = (t->capacity + 31) / 32;
        B2CO_CUDA(cudaMalloc(&t->d_newbits, 2 * words * 4));  // claimed bits, then shared bits
        B2CO_CUDA(cudaMalloc(&t->d_owner, t->capacity * 4));
        // owner entries stay all-ones between batches (each batch restores the ones it used)
        B2CO_CUDA(cudaMemset(t->d_owner, 0xff, t->capacity * 4));
        B2CO_CUDA(cudaStreamSynchronize(nullptr));  // done before any stream of the caller's uses it
    }
    if (t->pos_cap < n) {
        if (t->d_pos) cudaFree(t->d_pos);
        t->d_pos = nullptr;
        t->pos_cap = 0;
        B2CO_CUDA(cudaMalloc(&t->d_pos, n * 4));
        t->pos_cap = n;
    }
    return B2CO_OK;
}

}  // namespace

// First-wins InsertAndFind on scratch the caller provides: pos[n], two
// bitmaps of ceil(capacity/32) words (cleared here) and owner[capacity], whose
// entries must be all-ones on entry unless `owner_clear` is false (then they
// are set here); the call leaves them all-ones.
int b2co_oa_iaf_first_wins_on(b2co_oa_table* t, void const* pairs, void* out_found, uint8_t* out_inserted, uint64_t n,
                              uint32_t* pos, uint32_t* newbits, uint32_t* owner, bool owner_clear, cudaStream_t s)
{
    if (int st = check_table(t)) return st;
    if (int st = check_batch(n)) return st;
    B2CO_CUDA(cudaMemsetAsync(newbits, 0, ((t->capacity + 31) / 32) * 8, s));
    if (!owner_clear) B2CO_CUDA(cudaMemsetAsync(owner, 0xff, t->capacity * 4, s));
    return t->ops->iaf_first(t->args, t->desc.bucket_size, pairs, out_found, out_inserted, uint32_t(n), pos, newbits,
                             owner, s);
}

// Insert / InsertOrAssign with caller-owned device counters [failed, assigned]
// (zeroed by the caller), so concurrent launches on one table keep separate
// counts; nothing is synchronized.
int b2co_oa_launch_insert(b2co_oa_table* t, void const* pairs, uint64_t n, bool assign,
                          unsigned long long* d_counters, cudaStream_t s)
{
    if (int st = check_table(t)) return st;
    if (n == 0 || !pairs) return B2CO_OK;
    if (int st = check_batch(n)) return st;
    return t->ops->insert(t->args, t->desc.bucket_size, pairs, nullptr, uint32_t(n), assign, d_counters, s);
}

// Device bytes a table holds (slots and counters).
uint64_t b2co_oa_table_bytes(b2co_oa_table const* t)
{
    return t ? t->capacity * slot_bytes(t->desc.key_bytes, t->desc.value_bytes) + 3 * sizeof(unsigned long long) : 0;
}

// Key / payload / pair sizes of a table.
void b2co_oa_table_sizes(b2co_oa_table const* t, uint32_t* key_bytes, uint32_t* payload_bytes, uint32_t* pair_bytes)
{
    *key_bytes = t->desc.key_bytes;
    *payload_bytes = t->desc.value_bytes ? t->desc.value_bytes : t->desc.key_bytes;
    *pair_bytes = slot_bytes(t->desc.key_bytes, t->desc.value_bytes);
}

// Table creation with the clear optional: DynamicMap prepares its next submap
// uncleared and clears it on a side stream (the reference's DeferredClear
// constructor, include/static_map.h:611).
int b2co_oa_create_ex(b2co_oa_desc const* d, uint64_t requested, bool clear, b2co_stream stream,
                      b2co_oa_table** out)
{
    if (!d || !out) return fail(B2CO_EINVAL, "null descriptor or output");
    *out = nullptr;
    if (d->key_bytes != 2 && d->key_bytes != 4 && d->key_bytes != 8)
        return fail(B2CO_EINVAL, "key_bytes must be 2, 4 or 8");
    if (d->value_bytes != 0 && d->value_bytes != 2 && d->value_bytes != 4 && d->value_bytes != 8)
        return fail(B2CO_EINVAL, "value_bytes must be 0, 2, 4 or 8");
    if (d->probing > B2CO_PROBE_DOUBLE) return fail(B2CO_EINVAL, "unknown probing scheme");
    if (d->hash > B2CO_HASH_XXH64) return fail(B2CO_EINVAL, "unknown hash");
    if (d->key_kind > B2CO_KEY_FLOAT) return fail(B2CO_EINVAL, "unknown key kind");
    if (d->hash == B2CO_HASH_FMIX && d->key_bytes == 2)
        return fail(B2CO_EINVAL, "the Fmix hashes take 4- or 8-byte keys (hash_functions/utils.h:42-66)");
    if (!oa_ops_for(d->key_bytes, d->value_bytes, d->key_kind))
        return fail(B2CO_EINVAL, "unsupported key/payload layout (2-byte payloads need 2-byte keys; 2-byte keys take "
                                 "no payload or a 2-byte one)");
    uint64_t cap = 0;
    int st = b2co_oa_valid_capacity(requested, d->bucket_size, d->probing, &cap);
    if (st) return st;
    if (cap > 0xffffffffull)
        return fail(B2CO_ERANGE, "capacity exceeds the 32-bit slot index of the kernels");

    auto* t = new (std::nothrow) b2co_oa_table;
    if (!t) return fail(B2CO_ENOMEM, "host allocation failed");
    t->desc = *d;
    t->desc.empty_key_bits = mask_bytes(d->empty_key_bits, d->key_bytes);
    t->desc.erased_key_bits = mask_bytes(d->erased_key_bits, d->key_bytes);
    t->desc.empty_value_bits = mask_bytes(d->empty_value_bits, d->value_bytes ? d->value_bytes : 8);
    t->ops = oa_ops_for(d->key_bytes, d->value_bytes, d->key_kind);
    t->capacity = cap;
    cudaGetDevice(&t->device);
    default_shape(t);
    default_write_shape(t);

    uint32_t nb = uint32_t(cap / d->bucket_size);
    ProbeParams& p = t->args.probe;
    p.capacity = uint32_t(cap);
    p.nbuckets = nb;
    p.mod_nb = make_fastmod(nb);
    p.mod_nbm1 = make_fastmod(nb > 1 ? nb - 1 : 1);
    p.probing = d->probing;
    p.hash = d->hash;
    t->args.empty_key = t->desc.empty_key_bits;
    t->args.empty_value = d->value_bytes ? t->desc.empty_value_bits : 0;
    t->args.erased_key = t->desc.erased_key_bits;

    cudaError_t e = cudaMalloc(&t->args.slots, cap * slot_bytes(d->key_bytes, d->value_bytes));
    // counters: [failed, assigned, status word]
    if (e == cudaSuccess) e = cudaMalloc(&t->d_counters, 3 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(t->d_counters, 0, 3 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&t->h_counters, 3 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        b2co_oa_destroy(t);
        return cuda_fail(e, "table allocation");
    }
    if (clear && (st = b2co_oa_clear(t, stream))) {
        b2co_oa_destroy(t);
        return st;
    }
    *out = t;
    return B2CO_OK;
}

namespace {

__device__ unsigned long long g_gather_sink;

__device__ __forceinline__ uint32_t gather_mix(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Bare random bucket-window reads over a table's own 16- or 8-byte slots: the
// rate the first-window reads of a lookup can reach on this GPU, with none of a
// lookup's other work.  Four lanes per window and four windows in flight per
// lane group (the fastest form measured; one lane per 8-byte-slot window read
// 18.1 against 31.7 G windows/s); bucket b = mix(i ^ seed) % nbuckets, so every
// read stays inside the slot array.  Nothing is written but a sink word no real
// sum meets.
__device__ __forceinline__ unsigned long long fold_slot(U128 v) { return v.lo + v.hi; }
__device__ __forceinline__ unsigned long long fold_slot(unsigned long long v) { return v; }

template <int B, class W, int G>
__global__ void __launch_bounds__(256) k_window_gather(W const* slots, uint32_t nbuckets, uint32_t n, uint32_t seed)
{
    constexpr int K = 4, R = (B + G - 1) / G;
    uint32_t const r = threadIdx.x % G;
    uint32_t const groups = gridDim.x * (blockDim.x / G);
    uint32_t const g0 = blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
    unsigned long long acc = 0;
    for (uint32_t base = g0; base < n; base += groups * K) {
        W w[K][R];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            uint32_t const i = base + k * groups;
            uint32_t const idx = (gather_mix(i ^ seed) % nbuckets) * uint32_t(B);
#pragma unroll
            for (int s = 0; s < R; ++s)
                if (i < n && int(r) + s * G < B) w[k][s] = ld_ro(slots + idx + r + s * G);
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int s = 0; s < R; ++s)
                if (base + k * groups < n && int(r) + s * G < B) acc ^= fold_slot(w[k][s]);
    }
    if (acc == 0x9e3779b97f4a7c15ull) g_gather_sink = acc;  // keeps the reads live
}

}  // namespace

extern "C" {

int b2co_oa_window_gather(b2co_oa_table const* t, uint64_t n, uint32_t seed, b2co_stream stream)
{
    if (int st = check_table(t)) return st;
    uint32_t const sb = slot_bytes(t->desc.key_bytes, t->desc.value_bytes);
    if (sb != 16 && sb != 8) return fail(B2CO_EINVAL, "window gather needs 16- or 8-byte slots");
    if (n > (1ull << 31)) return fail(B2CO_ERANGE, "window gather: at most 2^31 windows per call");
    if (n == 0) return B2CO_OK;
    uint32_t const b = t->desc.bucket_size;
    uint32_t const nb = uint32_t(t->capacity / b);
    void const* k = nullptr;
    auto pick = [&](auto w) {
        using W = decltype(w);
        constexpr int G = 4;
        switch (b) {
        case 1: k = (void const*)k_window_gather<1, W, G>; break;
        case 2: k = (void const*)k_window_gather<2, W, G>; break;
        case 4: k = (void const*)k_window_gather<4, W, G>; break;
        case 5: k = (void const*)k_window_gather<5, W, G>; break;
        case 8: k = (void const*)k_window_gather<8, W, G>; break;
        default: break;
        }
    };
    if (sb == 16) pick(U128{});
    else pick(0ull);
    if (!k) return fail(B2CO_EINVAL, "unsupported bucket size");
    uint32_t grid = grid_for(k, 256, n, 64);
    void const* slots = t->args.slots;
    uint32_t n32 = uint32_t(n);
    void* params[] = {(void*)&slots, (void*)&nb, (void*)&n32, (void*)&seed};
    cudaError_t e = cudaLaunchKernel(k, dim3(grid), dim3(256), params, 0, cs(stream));
    return e == cudaSuccess ? B2CO_OK : cuda_fail(e, "window gather kernel");
}

int b2co_oa_create(b2co_oa_desc const* d, uint64_t requested, b2co_stream stream, b2co_oa_table** out)
{
    return b2co_oa_create_ex(d, requested, true, stream, out);
}

int b2co_oa_destroy(b2co_oa_table* t)
{
    if (!t) return B2CO_OK;
    if (t->args.slots) cudaFree(t->args.slots);
    if (t->d_counters) cudaFree(t->d_counters);
    if (t->h_counters) cudaFreeHost(t->h_counters);
    if (t->d_pos) cudaFree(t->d_pos);
    if (t->d_newbits) cudaFree(t->d_newbits);
    if (t->d_owner) cudaFree(t->d_owner);
    t->first_wins_order.release();
    if (t->stage) cudaFree(t->stage);
    for (auto& s : t->pipe)
        if (s) cudaStreamDestroy(s);
    for (auto& e : t->ev)
        if (e) cudaEventDestroy(e);
    delete t;
    return B2CO_OK;
}

int b2co_oa_capacity(b2co_oa_table const* t, uint64_t* c)
{
    if (int st = check_table(t)) return st;
    if (!c) return fail(B2CO_EINVAL, "null output");
    *c = t->capacity;
    return B2CO_OK;
}

int b2co_oa_data(b2co_oa_table const* t, void** slots)
{
    if (int st = check_table(t)) return st;
    if (!slots) return fail(B2CO_EINVAL, "null output");
    *slots = t->args.slots;
    return B2CO_OK;
}

int b2co_oa_describe(b2co_oa_table const* t, b2co_oa_desc* desc)
{
    if (int st = check_table(t)) return st;
    if (!desc) return fail(B2CO_EINVAL, "null output");
    *desc = t->desc;
    return B2CO_OK;
}

int b2co_oa_set_erased_key(b2co_oa_table* t, uint64_t erased, b2co_stream)
{
    if (int st = check_table(t)) return st;
    t->desc.erased_key_bits = mask_bytes(erased, t->desc.key_bytes);
    t->args.erased_key = t->desc.erased_key_bits;
    return B2CO_OK;
}

int b2co_oa_clear_async(b2co_oa_table* t, b2co_stream s)
{
    if (int st = check_table(t)) return st;
    return t->ops->clear(t->args, cs(s));
}

int b2co_oa_clear(b2co_oa_table* t, b2co_stream s)
{
    if (int st = b2co_oa_clear_async(t, s)) return st;
    B2CO_CUDA(cudaStreamSynchronize(cs(s)));
    return B2CO_OK;
}

// ---- inserts ---------------------------------------------------------------

static int insert_impl(b2co_oa_table* t, void const* pairs, uint8_t const* stencil, bool use_stencil, uint64_t n,
                       bool assign, b2co_stream s, uint64_t* failed, uint64_t* assigned)
{
    bool sync = failed != nullptr || assigned != nullptr;
    if (failed) *failed = 0;
    if (assigned) *assigned = 0;
    if (int st = check_table(t)) return st;
    if (n == 0) return B2CO_OK;
    if (!pairs || (use_stencil && !stencil)) {
        if (failed) *failed = n;
        return B2CO_OK;
    }
    if (int st = check_batch(n)) return st;
    cudaStream_t c = cs(s);
    if (sync) B2CO_CUDA(cudaMemsetAsync(t->d_counters, 0, 2 * sizeof(unsigned long long), c));
    int st = t->ops->insert(t->args, t->desc.bucket_size, pairs, stencil, uint32_t(n), assign,
                            sync ? t->d_counters : nullptr, c);
    if (st || !sync) return st;
    if ((st = sync_counters(t, c, 2))) return st;
    if (failed) *failed = t->h_counters[0];
    if (assigned) *assigned = t->h_counters[1];
    return B2CO_OK;
}

int b2co_oa_insert(b2co_oa_table* t, void const* pairs, uint64_t n, b2co_stream s, uint64_t* failed)
{
    uint64_t dummy;
    return insert_impl(t, pairs, nullptr, false, n, false, s, failed ? failed : &dummy, nullptr);
}

int b2co_oa_insert_async(b2co_oa_table* t, void const* pairs, uint64_t n, b2co_stream s)
{
    return insert_impl(t, pairs, nullptr, false, n, false, s, nullptr, nullptr);
}

int b2co_oa_insert_if(b2co_oa_table* t, void const* pairs, uint8_t const* stencil, uint64_t n, b2co_stream s,
                      uint64_t* failed)
{
    uint64_t dummy;
    return insert_impl(t, pairs, stencil, true, n, false, s, failed ? failed : &dummy, nullptr);
}

int b2co_oa_insert_if_async(b2co_oa_table* t, void const* pairs, uint8_t const* stencil, uint64_t n, b2co_stream s)
{
    return insert_impl(t, pairs, stencil, true, n, false, s, nullptr, nullptr);
}

int b2co_oa_insert_or_assign(b2co_oa_table* t, void const* pairs, uint64_t n, b2co_stream s, uint64_t* failed,
                             uint64_t* assigned)
{
    uint64_t f, a;
    if (t && t->desc.value_bytes == 0) return fail(B2CO_EINVAL, "InsertOrAssign needs a map (value_bytes > 0)");
    return insert_impl(t, pairs, nullptr, false, n, true, s, failed ? failed : &f, assigned ? assigned : &a);
}

int b2co_oa_insert_or_assign_async(b2co_oa_table* t, void const* pairs, uint64_t n, b2co_stream s)
{
    if (t && t->desc.value_bytes == 0) return fail(B2CO_EINVAL, "InsertOrAssign needs a map (value_bytes > 0)");
    return insert_impl(t, pairs, nullptr, false, n, true, s, nullptr, nullptr);
}

int b2co_oa_assign_if_async(b2co_oa_table* t, void const* pairs, uint8_t const* stencil, uint64_t n, b2co_stream s)
{
    if (int st = check_table(t)) return st;
    if (t->desc.value_bytes == 0) return fail(B2CO_EINVAL, "AssignIf needs a map (value_bytes > 0)");
    if (n == 0 || !pairs || !stencil) return B2CO_OK;
    if (int st = check_batch(n)) return st;
    return t->ops->assign_if(t->args, t->desc.bucket_size, pairs, stencil, uint32_t(n), cs(s));
}

int b2co_oa_insert_and_find_async(b2co_oa_table* t, void const* pairs, void* out_found, uint8_t* out_inserted,
                                  uint64_t n, int mode, b2co_stream s)
{
    if (int st = check_table(t)) return st;
    if (n == 0 || !pairs) return B2CO_OK;
    if (!out_found || !out_inserted) return fail(B2CO_EINVAL, "InsertAndFind outputs must not be null");
    if (int st = check_batch(n)) return st;
    if (mode == B2CO_IAF_RACE)
        return t->ops->iaf_race(t->args, t->desc.bucket_size, pairs, out_found, out_inserted, uint32_t(n), cs(s));
    if (mode != B2CO_IAF_FIRST_WINS) return fail(B2CO_EINVAL, "unknown InsertAndFind mode");
    if (int st = ensure_first_wins_scratch(t, n)) return st;
    if (int st = t->first_wins_order.begin(cs(s))) return st;
    B2CO_CUDA(cudaMemsetAsync(t->d_newbits, 0, ((t->capacity + 31) / 32) * 8, cs(s)));
    if (int st = t->ops->iaf_first(t->args, t->desc.bucket_size, pairs, out_found, out_inserted, uint32_t(n),
                                   t->d_pos, t->d_newbits, t->d_owner, cs(s)))
        return st;
    return t->first_wins_order.end(cs(s));
}

int b2co_oa_reserve_insert_and_find(b2co_oa_table* t, uint64_t n)
{
    if (int st = check_table(t)) return st;
    if (int st = check_batch(n)) return st;
    return ensure_first_wins_scratch(t, n ? n : 1);
}

int b2co_oa_insert_and_find(b2co_oa_table* t, void const* pairs, void* out_found, uint8_t* out_inserted, uint64_t n,
                            int mode, b2co_stream s)
{
    if (int st = b2co_oa_insert_and_find_async(t, pairs, out_found, out_inserted, n, mode, s)) return st;
    B2CO_CUDA(cudaStreamSynchronize(cs(s)));
    return B2CO_OK;
}

// ---- erase / count ---------------------------------------------------------

static int erase_impl(b2co_oa_table* t, void const* keys, uint64_t n, b2co_stream s, uint64_t* failed)
{
    if (failed) *failed = 0;
    if (int st = check_table(t)) return st;
    if (n == 0) return B2CO_OK;
    if (!keys) {
        if (failed) *failed = n;
        return B2CO_OK;
    }
    if (int st = check_batch(n)) return st;
    cudaStream_t c = cs(s);
    if (failed) B2CO_CUDA(cudaMemsetAsync(t->d_counters, 0, sizeof(unsigned long long), c));
    int st = t->ops->erase(t->args, t->desc.bucket_size, keys, uint32_t(n), failed ? t->d_counters : nullptr, c);
    if (st || !failed) return st;
    if ((st = sync_counters(t, c, 1))) return st;
    *failed = t->h_counters[0];
    return B2CO_OK;
}

int b2co_oa_erase(b2co_oa_table* t, void const* keys, uint64_t n, b2co_stream s, uint64_t* failed)
{
    uint64_t dummy;
    return erase_impl(t, keys, n, s, failed ? failed : &dummy);
}

int b2co_oa_erase_async(b2co_oa_table* t, void const* keys, uint64_t n, b2co_stream s)
{
    return erase_impl(t, keys, n, s, nullptr);
}

int b2co_oa_count(b2co_oa_table* t, void const* keys, uint64_t n, b2co_stream s, uint64_t* count)
{
    if (!count) return fail(B2CO_EINVAL, "null output");
    *count = 0;
    if (int st = check_table(t)) return st;
    if (n == 0 || !keys) return B2CO_OK;
    if (int st = check_batch(n)) return st;
    cudaStream_t c = cs(s);
    B2CO_CUDA(cudaMemsetAsync(t->d_counters, 0, sizeof(unsigned long long), c));
    int st = t->ops->count(t->args, t->desc.bucket_size, keys, uint32_t(n), t->d_counters, c);
    if (st) return st;
    if ((st = sync_counters(t, c, 1))) return st;
    *count = t->h_counters[0];
    return B2CO_OK;
}

// ---- lookups -----------------------------------------------------------------

static int lookup_async(b2co_oa_table* t, bool contains, void const* keys, uint8_t const* stencil, bool use_stencil,
                        void* out, uint64_t n, b2co_stream s)
{
    if (int st = check_table(t)) return st;
    if (n == 0 || !keys || !out || (use_stencil && !stencil)) return B2CO_OK;
    if (int st = check_batch(n)) return st;
    return launch_find(t, contains, keys, stencil, out, n, cs(s));
}

static int lookup_sync(b2co_oa_table* t, bool contains, void const* keys, uint8_t const* stencil, bool use_stencil,
                       void* out, uint64_t n, b2co_stream s)
{
    if (int st = lookup_async(t, contains, keys, stencil, use_stencil, out, n, s)) return st;
    return check_status(t, cs(s));
}

int b2co_oa_find(b2co_oa_table* t, void const* k, void* o, uint64_t n, b2co_stream s)
{
    return lookup_sync(t, false, k, nullptr, false, o, n, s);
}
int b2co_oa_find_async(b2co_oa_table* t, void const* k, void* o, uint64_t n, b2co_stream s)
{
    return lookup_async(t, false, k, nullptr, false, o, n, s);
}
int b2co_oa_find_if(b2co_oa_table* t, void const* k, uint8_t const* st, void* o, uint64_t n, b2co_stream s)
{
    return lookup_sync(t, false, k, st, true, o, n, s);
}
int b2co_oa_find_if_async(b2co_oa_table* t, void const* k, uint8_t const* st, void* o, uint64_t n, b2co_stream s)
{
    return lookup_async(t, false, k, st, true, o, n, s);
}
int b2co_oa_contains(b2co_oa_table* t, void const* k, uint8_t* o, uint64_t n, b2co_stream s)
{
    return lookup_sync(t, true, k, nullptr, false, o, n, s);
}
int b2co_oa_contains_async(b2co_oa_table* t, void const* k, uint8_t* o, uint64_t n, b2co_stream s)
{
    return lookup_async(t, true, k, nullptr, false, o, n, s);
}
int b2co_oa_contains_if(b2co_oa_table* t, void const* k, uint8_t const* st, uint8_t* o, uint64_t n, b2co_stream s)
{
    return lookup_sync(t, true, k, st, true, o, n, s);
}
int b2co_oa_contains_if_async(b2co_oa_table* t, void const* k, uint8_t const* st, uint8_t* o, uint64_t n,
                              b2co_stream s)
{
    return lookup_async(t, true, k, st, true, o, n, s);
}

int b2co_oa_set_find_shape(b2co_oa_table* t, uint32_t lanes, uint32_t items)
{
    if (int st = check_table(t)) return st;
    if (lanes == 0 && items == 0) {
        default_shape(t);
        return B2CO_OK;
    }
    if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8) return fail(B2CO_EINVAL, "lanes must be 1, 2, 4 or 8");
    uint32_t const k = items & ~(kShapeSegmented | kShapeBulk | kShapeWarpStaged | kShapeDeferred);
    if (k != 1 && k != 2 && k != 4) return fail(B2CO_EINVAL, "keys per lane must be 1, 2 or 4");
    t->find_lanes = lanes;
    t->find_items = items;
    return B2CO_OK;
}

int b2co_oa_set_write_shape(b2co_oa_table* t, uint32_t lanes, uint32_t keys_per_tile)
{
    if (int st = check_table(t)) return st;
    if (lanes == 0 && keys_per_tile == 0) {
        default_write_shape(t);
        return B2CO_OK;
    }
    if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8) return fail(B2CO_EINVAL, "lanes must be 1, 2, 4 or 8");
    if (keys_per_tile != 1 && keys_per_tile != 2 && keys_per_tile != 4)
        return fail(B2CO_EINVAL, "keys per lane group must be 1, 2 or 4");
    t->args.write_shape = (lanes << 8) | keys_per_tile;
    return B2CO_OK;
}

// Host-buffer Find: chunks of up to 4 Mi keys rotate over kHostSlots staging
// slots, one pipeline stream per slot, each chunk copy-in -> probe -> copy-out in
// its stream.  Consecutive chunks sit on different streams, so later chunks copy
// in while earlier ones probe and copy out and both copy directions stay busy.
// Only the first copy-in and the last copy-out run with the other direction
// idle, so a batch of 16 Mi keys or more starts with chunks of 1 and 2 Mi keys
// and ends with 2 and 1 Mi (uniform 1 or 2 Mi chunks measured slower: each
// chunk costs about 40 us of pipeline overhead).  Pinned host buffers give full
// overlap.
constexpr uint64_t kHostChunk = 1ull << 22;  // keys per full chunk

static uint64_t host_chunk_at(uint64_t off, uint64_t n)
{
    uint64_t const q = kHostChunk / 4, h = kHostChunk / 2, left = n - off;
    if (n < 4 * kHostChunk) return left < kHostChunk ? left : kHostChunk;
    if (off == 0) return q;
    if (off == q) return h;
    if (left <= q) return left;
    if (left <= q + h) return left - q;                       // then the last quarter
    if (left <= q + h + kHostChunk) return left - q - h;      // then a half and a quarter
    return kHostChunk;
}
int b2co_oa_find_host(b2co_oa_table* t, void const* host_keys, void* host_out, uint64_t n, b2co_stream s)
{
    if (int st = check_table(t)) return st;
    if (n == 0 || !host_keys || !host_out) return B2CO_OK;
    uint32_t const kb = t->desc.key_bytes;
    uint32_t const ob = t->desc.value_bytes ? t->desc.value_bytes : kb;
    uint64_t const chunk = kHostChunk;
    if (!t->stage) {
        t->stage_keys = chunk;
        B2CO_CUDA(cudaMalloc(&t->stage, kHostSlots * chunk * (kb + ob)));
        for (auto& p : t->pipe) B2CO_CUDA(cudaStreamCreateWithFlags(&p, cudaStreamNonBlocking));
        for (auto& e : t->ev) B2CO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaStream_t c = cs(s);
    B2CO_CUDA(cudaEventRecord(t->ev[kHostSlots], c));
    for (auto& p : t->pipe) B2CO_CUDA(cudaStreamWaitEvent(p, t->ev[kHostSlots], 0));
    char* base = static_cast<char*>(t->stage);
    for (uint64_t off = 0, c_i = 0, m = 0; off < n; off += m, ++c_i) {
        m = host_chunk_at(off, n);
        int slot = int(c_i % kHostSlots);
        cudaStream_t p = t->pipe[slot];
        char* dk = base + uint64_t(slot) * chunk * (kb + ob);
        char* dout = dk + chunk * kb;
        B2CO_CUDA(cudaMemcpyAsync(dk, static_cast<char const*>(host_keys) + off * kb, m * kb,
                                  cudaMemcpyHostToDevice, p));
        if (int st = launch_find(t, false, dk, nullptr, dout, m, p)) return st;
        B2CO_CUDA(cudaMemcpyAsync(static_cast<char*>(host_out) + off * ob, dout, m * ob, cudaMemcpyDeviceToHost, p));
    }
    for (int i = 0; i < kHostSlots; ++i) {
        B2CO_CUDA(cudaEventRecord(t->ev[i], t->pipe[i]));
        B2CO_CUDA(cudaStreamWaitEvent(c, t->ev[i], 0));
    }
    return check_status(t, c);
}

}  // extern "C"
