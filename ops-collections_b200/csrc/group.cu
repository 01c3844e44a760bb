// group.cu -- C ABI of table groups: many independent StaticMap/StaticSet
// tables of uneven sizes served by one persistent launch (the batched
// pattern: per-partition group-by / join builds).
//
// Every table keeps the single-table semantics (capacity from the prime rule,
// probing, sentinels); the group only packs them into one slab with a device
// array of per-table descriptors, and runs each operation over all tables in
// one launch -- optionally replayed from a CUDA graph -- instead of one launch
// per table.  The per-table launch path is kept as the baseline to beat.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "b2co_host.h"
#include "group_kernels.cuh"

using namespace b2co;

struct b2co_oa_group {
    b2co_oa_desc desc{};
    GroupOps const* gops = nullptr;
    OaOps const* ops = nullptr;
    uint32_t count = 0;
    uint32_t slot_bytes = 0;
    std::vector<GroupTable> host_tables;
    void* slab = nullptr;
    uint64_t total_slots = 0;
    GroupTable* d_tables = nullptr;
    unsigned long long* d_counters = nullptr;  // [failed, status]
    unsigned long long* h_counters = nullptr;
    uint32_t find_shape = 4u | (2u << 8);  // lanes | keys per lane group << 8 | block << 16 (0 = 256)
    // one cached graph of the group Find launch
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    void const* g_keys = nullptr;
    void const* g_offsets = nullptr;
    void* g_out = nullptr;
    uint64_t g_n = 0;
    uint32_t g_shape = 0;
    bool g_contains = false;
};

namespace {

cudaStream_t cs(b2co_stream s) { return reinterpret_cast<cudaStream_t>(s); }

OaOps const* ops_for(uint32_t kb, uint32_t vb, GroupOps const** g)
{
    if (kb == 4 && vb == 0) return *g = &kGroupSet4, &kOpsSet4;
    if (kb == 8 && vb == 0) return *g = &kGroupSet8, &kOpsSet8;
    if (kb == 4 && vb == 4) return *g = &kGroupMap44, &kOpsMap44;
    if (kb == 4 && vb == 8) return *g = &kGroupMap48, &kOpsMap48;
    if (kb == 8 && vb == 4) return *g = &kGroupMap84, &kOpsMap84;
    if (kb == 8 && vb == 8) return *g = &kGroupMap88, &kOpsMap88;
    return nullptr;
}

uint64_t mask_bytes(uint64_t v, uint32_t n) { return n >= 8 ? v : (v & ((1ull << (8 * n)) - 1ull)); }

GroupArgs group_args(b2co_oa_group const* g, uint64_t const* d_offsets)
{
    GroupArgs a;
    a.slots = g->slab;
    a.tables = g->d_tables;
    a.offsets = d_offsets;
    a.count = g->count;
    a.empty_key = g->desc.empty_key_bits;
    a.empty_value = g->desc.value_bytes ? g->desc.empty_value_bits : 0;
    return a;
}

OaArgs table_args(b2co_oa_group const* g, uint32_t t)
{
    OaArgs a{};
    a.slots = static_cast<char*>(g->slab) + g->host_tables[t].slot_offset * g->slot_bytes;
    a.probe = g->host_tables[t].probe;
    a.empty_key = g->desc.empty_key_bits;
    a.empty_value = g->desc.value_bytes ? g->desc.empty_value_bits : 0;
    a.erased_key = g->desc.empty_key_bits;
    return a;
}

int check(b2co_oa_group const* g)
{
    if (!g || !g->slab) return fail(B2CO_ELOGIC, "table group is null or has no storage");
    return B2CO_OK;
}

// ---- autotune cache ----------------------------------------------------------
// Keyed by (op, key bytes, payload bytes, bucket size, capacity bucket); the
// value is a packed kernel shape and the time it measured.
struct TuneKey {
    uint32_t op, kb, vb, b, cap_bucket;
    bool operator<(TuneKey const& o) const
    {
        return std::tie(op, kb, vb, b, cap_bucket) < std::tie(o.op, o.kb, o.vb, o.b, o.cap_bucket);
    }
};
struct TuneVal {
    uint32_t shape;
    float ms;
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;
bool g_tune_env_loaded = false;

uint32_t capacity_bucket(uint64_t mean_capacity)
{
    uint32_t b = 0;
    while (mean_capacity > 1) mean_capacity >>= 1, ++b;
    return b;
}

int load_file_locked(char const* path)
{
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(B2CO_EINVAL, std::string("cannot read the tune cache ") + path);
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
        char op[32];
        TuneKey k{};
        unsigned lanes, items, block;
        float ms;
        if (std::sscanf(line, "%31s %u %u %u %u %u %u %u %f", op, &k.kb, &k.vb, &k.b, &k.cap_bucket, &lanes, &items,
                        &block, &ms) != 9 || std::strcmp(op, "group_find") != 0)
            continue;  // comments and unknown operations
        g_tune[k] = TuneVal{lanes | (items << 8) | (block << 16), ms};
    }
    std::fclose(f);
    return B2CO_OK;
}

int save_file_locked(char const* path)
{
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(B2CO_EINVAL, std::string("cannot write the tune cache ") + path);
    std::fprintf(f, "# op key_bytes payload_bytes bucket log2_capacity lanes keys_per_tile block ms\n");
    for (auto const& kv : g_tune) {
        TuneKey const& k = kv.first;
        uint32_t const sh = kv.second.shape;
        std::fprintf(f, "group_find %u %u %u %u %u %u %u %.4f\n", k.kb, k.vb, k.b, k.cap_bucket, sh & 0xffu,
                     (sh >> 8) & 0xffu, (sh >> 16) ? (sh >> 16) : 256u, kv.second.ms);
    }
    std::fclose(f);
    return B2CO_OK;
}

void env_load_locked()
{
    if (g_tune_env_loaded) return;
    g_tune_env_loaded = true;
    if (char const* p = std::getenv("B2CO_TUNE_CACHE")) {
        if (FILE* f = std::fopen(p, "r")) {
            std::fclose(f);
            load_file_locked(p);
        }
    }
}

bool tune_cache_get(TuneKey const& k, uint32_t* shape)
{
    std::lock_guard<std::mutex> l(g_tune_mu);
    env_load_locked();
    auto it = g_tune.find(k);
    if (it == g_tune.end()) return false;
    *shape = it->second.shape;
    return true;
}

void tune_cache_put(TuneKey const& k, uint32_t shape, float ms)
{
    std::lock_guard<std::mutex> l(g_tune_mu);
    env_load_locked();
    g_tune[k] = TuneVal{shape, ms};
    if (char const* p = std::getenv("B2CO_TUNE_CACHE")) save_file_locked(p);
}

}  // namespace

extern "C" {

int b2co_oa_group_create(b2co_oa_desc const* d, uint64_t const* requested, uint32_t count, b2co_stream stream,
                         b2co_oa_group** out)
{
    if (!d || !requested || !out) return fail(B2CO_EINVAL, "null argument");
    *out = nullptr;
    if (count == 0) return fail(B2CO_EINVAL, "a table group needs at least one table");
    GroupOps const* gops = nullptr;
    OaOps const* ops = ops_for(d->key_bytes, d->value_bytes, &gops);
    if (!ops) return fail(B2CO_EINVAL, "unsupported key/value sizes");
    if (d->probing > B2CO_PROBE_DOUBLE || d->hash > B2CO_HASH_XXH64)
        return fail(B2CO_EINVAL, "bad descriptor");
    if (d->key_kind != B2CO_KEY_INTEGER) return fail(B2CO_EINVAL, "table groups take integer keys");
    auto* g = new (std::nothrow) b2co_oa_group;
    if (!g) return fail(B2CO_ENOMEM, "host allocation failed");
    std::unique_ptr<b2co_oa_group, int (*)(b2co_oa_group*)> guard(g, b2co_oa_group_destroy);
    g->desc = *d;
    g->desc.empty_key_bits = mask_bytes(d->empty_key_bits, d->key_bytes);
    g->desc.empty_value_bits = mask_bytes(d->empty_value_bits, d->value_bytes ? d->value_bytes : 8);
    g->ops = ops;
    g->gops = gops;
    g->count = count;
    g->slot_bytes = d->value_bytes == 0 ? d->key_bytes : (d->key_bytes + d->value_bytes == 8 ? 8 : 16);
    g->host_tables.resize(count);
    uint64_t off = 0;
    for (uint32_t t = 0; t < count; ++t) {
        uint64_t cap = 0;
        if (int st = b2co_oa_valid_capacity(requested[t], d->bucket_size, d->probing, &cap)) return st;
        if (cap > 0xffffffffull) return fail(B2CO_ERANGE, "table capacity exceeds the 32-bit slot index");
        GroupTable& gt = g->host_tables[t];
        gt.slot_offset = off;
        uint32_t nb = uint32_t(cap / d->bucket_size);
        gt.probe.capacity = uint32_t(cap);
        gt.probe.nbuckets = nb;
        gt.probe.mod_nb = make_fastmod(nb);
        gt.probe.mod_nbm1 = make_fastmod(nb > 1 ? nb - 1 : 1);
        gt.probe.probing = d->probing;
        gt.probe.hash = d->hash;
        off += cap;
    }
    g->total_slots = off;
    B2CO_CUDA(cudaMalloc(&g->slab, off * g->slot_bytes));
    B2CO_CUDA(cudaMalloc(&g->d_tables, sizeof(GroupTable) * count));
    B2CO_CUDA(cudaMemcpy(g->d_tables, g->host_tables.data(), sizeof(GroupTable) * count, cudaMemcpyHostToDevice));
    B2CO_CUDA(cudaMalloc(&g->d_counters, 2 * sizeof(unsigned long long)));
    B2CO_CUDA(cudaMemset(g->d_counters, 0, 2 * sizeof(unsigned long long)));
    B2CO_CUDA(cudaMallocHost(&g->h_counters, 2 * sizeof(unsigned long long)));
    B2CO_CUDA(cudaStreamCreateWithFlags(&g->capture_stream, cudaStreamNonBlocking));
    if (int st = b2co_oa_group_clear(g, stream)) return st;
    *out = guard.release();
    return B2CO_OK;
}

int b2co_oa_group_destroy(b2co_oa_group* g)
{
    if (!g) return B2CO_OK;
    if (g->graph) cudaGraphExecDestroy(g->graph);
    if (g->capture_stream) cudaStreamDestroy(g->capture_stream);
    if (g->slab) cudaFree(g->slab);
    if (g->d_tables) cudaFree(g->d_tables);
    if (g->d_counters) cudaFree(g->d_counters);
    if (g->h_counters) cudaFreeHost(g->h_counters);
    delete g;
    return B2CO_OK;
}

int b2co_oa_group_table_capacity(b2co_oa_group const* g, uint32_t t, uint64_t* cap)
{
    if (int st = check(g)) return st;
    if (!cap || t >= g->count) return fail(B2CO_EINVAL, "bad table index or null output");
    *cap = g->host_tables[t].probe.capacity;
    return B2CO_OK;
}

int b2co_oa_group_total_slots(b2co_oa_group const* g, uint64_t* slots)
{
    if (int st = check(g)) return st;
    if (!slots) return fail(B2CO_EINVAL, "null output");
    *slots = g->total_slots;
    return B2CO_OK;
}

int b2co_oa_group_data(b2co_oa_group const* g, void** slab)
{
    if (int st = check(g)) return st;
    if (!slab) return fail(B2CO_EINVAL, "null output");
    *slab = g->slab;
    return B2CO_OK;
}

int b2co_oa_group_clear(b2co_oa_group* g, b2co_stream s)
{
    if (int st = check(g)) return st;
    // the clear kernel indexes slots in 32 bits: clear the slab in pieces
    uint64_t const piece = 1ull << 31;
    for (uint64_t off = 0; off < g->total_slots; off += piece) {
        OaArgs a{};
        a.slots = static_cast<char*>(g->slab) + off * g->slot_bytes;
        uint64_t m = g->total_slots - off < piece ? g->total_slots - off : piece;
        a.probe.capacity = uint32_t(m);
        a.empty_key = g->desc.empty_key_bits;
        a.empty_value = g->desc.value_bytes ? g->desc.empty_value_bits : 0;
        if (int st = g->ops->clear(a, cs(s))) return st;
    }
    B2CO_CUDA(cudaStreamSynchronize(cs(s)));
    return B2CO_OK;
}

// Insert into every table in one launch; pairs of table t are
// [offsets[t], offsets[t+1]) of the concatenation (device offsets, count + 1).
int b2co_oa_group_insert(b2co_oa_group* g, void const* pairs, uint64_t const* d_offsets, uint64_t n, b2co_stream s,
                         uint64_t* failed)
{
    if (failed) *failed = 0;
    if (int st = check(g)) return st;
    if (n == 0 || !pairs) return B2CO_OK;
    if (!d_offsets) return fail(B2CO_EINVAL, "offsets must not be null");
    cudaStream_t c = cs(s);
    if (failed) B2CO_CUDA(cudaMemsetAsync(g->d_counters, 0, sizeof(unsigned long long), c));
    int st = g->gops->insert(group_args(g, d_offsets), g->desc.bucket_size, pairs, n, failed ? g->d_counters : nullptr, c);
    if (st || !failed) return st;
    B2CO_CUDA(cudaMemcpyAsync(g->h_counters, g->d_counters, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c));
    B2CO_CUDA(cudaStreamSynchronize(c));
    *failed = g->h_counters[0];
    return B2CO_OK;
}

int b2co_oa_group_find(b2co_oa_group* g, void const* keys, uint64_t const* d_offsets, void* out, uint64_t n,
                       int contains, b2co_stream s)
{
    if (int st = check(g)) return st;
    if (n == 0 || !keys || !out) return B2CO_OK;
    if (!d_offsets) return fail(B2CO_EINVAL, "offsets must not be null");
    return g->gops->find(group_args(g, d_offsets), g->desc.bucket_size, g->find_shape, contains != 0, keys, out, n,
                         cs(s));
}

// The same launch replayed from a CUDA graph captured on first use (and again
// whenever the arguments or the lane count change).
int b2co_oa_group_find_graph(b2co_oa_group* g, void const* keys, uint64_t const* d_offsets, void* out, uint64_t n,
                             int contains, b2co_stream s)
{
    if (int st = check(g)) return st;
    if (n == 0 || !keys || !out) return B2CO_OK;
    if (!d_offsets) return fail(B2CO_EINVAL, "offsets must not be null");
    bool const same = g->graph && g->g_keys == keys && g->g_offsets == d_offsets && g->g_out == out && g->g_n == n &&
                      g->g_shape == g->find_shape && g->g_contains == (contains != 0);
    if (!same) {
        if (g->graph) {
            cudaGraphExecDestroy(g->graph);
            g->graph = nullptr;
        }
        B2CO_CUDA(cudaStreamBeginCapture(g->capture_stream, cudaStreamCaptureModeThreadLocal));
        int st = g->gops->find(group_args(g, d_offsets), g->desc.bucket_size, g->find_shape, contains != 0, keys, out,
                               n, g->capture_stream);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(g->capture_stream, &graph);
        if (st) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&g->graph, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        g->g_keys = keys;
        g->g_offsets = d_offsets;
        g->g_out = out;
        g->g_n = n;
        g->g_shape = g->find_shape;
        g->g_contains = contains != 0;
    }
    B2CO_CUDA(cudaGraphLaunch(g->graph, cs(s)));
    return B2CO_OK;
}

// Baseline: one plain launch per table, each on its slice (host offsets).
int b2co_oa_group_find_per_table(b2co_oa_group* g, void const* keys, uint64_t const* h_offsets, void* out,
                                 int contains, b2co_stream s)
{
    if (int st = check(g)) return st;
    if (!keys || !out || !h_offsets) return fail(B2CO_EINVAL, "null argument");
    uint32_t const kb = g->desc.key_bytes, ob = contains ? 1 : (g->desc.value_bytes ? g->desc.value_bytes : kb);
    for (uint32_t t = 0; t < g->count; ++t) {
        uint64_t const lo = h_offsets[t], m = h_offsets[t + 1] - lo;
        if (m == 0) continue;
        int st = g->ops->find(table_args(g, t), g->desc.bucket_size, 2, 2, contains != 0,
                              static_cast<char const*>(keys) + lo * kb, nullptr, static_cast<char*>(out) + lo * ob,
                              uint32_t(m), wait_ctl(reinterpret_cast<unsigned int*>(g->d_counters + 1)), cs(s));
        if (st) return st;
    }
    return B2CO_OK;
}

int b2co_oa_group_insert_per_table(b2co_oa_group* g, void const* pairs, uint64_t const* h_offsets, b2co_stream s)
{
    if (int st = check(g)) return st;
    if (!pairs || !h_offsets) return fail(B2CO_EINVAL, "null argument");
    for (uint32_t t = 0; t < g->count; ++t) {
        uint64_t const lo = h_offsets[t], m = h_offsets[t + 1] - lo;
        if (m == 0) continue;
        int st = g->ops->insert(table_args(g, t), g->desc.bucket_size, static_cast<char const*>(pairs) + lo * g->slot_bytes,
                                nullptr, uint32_t(m), false, nullptr, cs(s));
        if (st) return st;
    }
    return B2CO_OK;
}

int b2co_oa_group_set_find_shape_ex(b2co_oa_group* g, uint32_t lanes, uint32_t keys_per_tile, uint32_t block)
{
    if (int st = check(g)) return st;
    if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8) return fail(B2CO_EINVAL, "lanes must be 1, 2, 4 or 8");
    if (keys_per_tile != 1 && keys_per_tile != 2 && keys_per_tile != 4)
        return fail(B2CO_EINVAL, "keys per lane group must be 1, 2 or 4");
    if (keys_per_tile > lanes && lanes > 1) return fail(B2CO_EINVAL, "keys per lane group cannot exceed the lanes");
    if (block != 0 && block != 64 && block != 128 && block != 256)
        return fail(B2CO_EINVAL, "threads per block must be 64, 128 or 256");
    g->find_shape = lanes | (keys_per_tile << 8) | (block << 16);
    return B2CO_OK;
}

int b2co_oa_group_set_find_shape(b2co_oa_group* g, uint32_t lanes)
{
    return b2co_oa_group_set_find_shape_ex(g, lanes, 1, 0);
}

int b2co_oa_group_get_find_shape(b2co_oa_group const* g, uint32_t* lanes, uint32_t* keys_per_tile, uint32_t* block)
{
    if (int st = check(g)) return st;
    if (lanes) *lanes = g->find_shape & 0xffu;
    if (keys_per_tile) *keys_per_tile = (g->find_shape >> 8) & 0xffu;
    if (block) *block = (g->find_shape >> 16) ? (g->find_shape >> 16) : 256u;
    return B2CO_OK;
}

// Autotuner: times the group Find with every kernel shape -- lanes per window,
// keys in flight per lane group, threads per block -- on the caller's own
// batch and keeps the fastest.  Results are cached in the process under (op,
// key bytes, payload bytes, bucket size, log2 of the mean table capacity) and
// reused without timing; the cache can be saved to and loaded from a file
// (b2co_tune_cache_save / _load, or the B2CO_TUNE_CACHE file, loaded on first
// use and rewritten after each new result).  Outputs are overwritten with
// valid results.
int b2co_oa_group_autotune(b2co_oa_group* g, void const* keys, uint64_t const* d_offsets, void* out, uint64_t n,
                           b2co_stream s, uint32_t* lanes, uint32_t* keys_per_tile, uint32_t* block, int* from_cache)
{
    if (int st = check(g)) return st;
    if (n == 0 || !keys || !out || !d_offsets) return fail(B2CO_EINVAL, "autotune needs a non-empty batch");
    TuneKey const key{0, g->desc.key_bytes, g->desc.value_bytes, g->desc.bucket_size,
                      capacity_bucket(g->total_slots / g->count)};
    uint32_t shape = 0;
    bool const hit = tune_cache_get(key, &shape);
    if (!hit) {
        cudaStream_t c = cs(s);
        cudaEvent_t e0, e1;
        B2CO_CUDA(cudaEventCreate(&e0));
        B2CO_CUDA(cudaEventCreate(&e1));
        float best = 1e30f;
        uint32_t const saved = g->find_shape;
        shape = saved;
        static uint32_t const kLanes[] = {1, 2, 4, 8}, kItems[] = {1, 2, 4}, kBlocks[] = {128, 256};
        int st = B2CO_OK;
        for (uint32_t ln : kLanes) {
            for (uint32_t it : kItems) {
                if ((ln == 1 && it > 1) || (ln > 1 && it > ln)) continue;
                for (uint32_t bl : kBlocks) {
                    g->find_shape = ln | (it << 8) | (bl << 16);
                    if ((st = b2co_oa_group_find(g, keys, d_offsets, out, n, 0, s))) break;  // warm
                    cudaEventRecord(e0, c);
                    for (int r = 0; r < 3 && !st; ++r) st = b2co_oa_group_find(g, keys, d_offsets, out, n, 0, s);
                    cudaEventRecord(e1, c);
                    cudaEventSynchronize(e1);
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (st) break;
                    if (ms < best) best = ms, shape = g->find_shape;
                }
                if (st) break;
            }
            if (st) break;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st) {
            g->find_shape = saved;
            return st;
        }
        tune_cache_put(key, shape, best / 3.0f);
    }
    g->find_shape = shape;
    if (from_cache) *from_cache = hit ? 1 : 0;
    b2co_oa_group_get_find_shape(g, lanes, keys_per_tile, block);
    return b2co_oa_group_find(g, keys, d_offsets, out, n, 0, s);
}

// The lanes-only form of the autotuner (the shape it picks is kept whole).
int b2co_oa_group_autotune_find(b2co_oa_group* g, void const* keys, uint64_t const* d_offsets, void* out, uint64_t n,
                                b2co_stream s, uint32_t* chosen_lanes)
{
    return b2co_oa_group_autotune(g, keys, d_offsets, out, n, s, chosen_lanes, nullptr, nullptr, nullptr);
}

}  // extern "C"

extern "C" {

int b2co_tune_cache_save(char const* path)
{
    if (!path) return fail(B2CO_EINVAL, "null path");
    std::lock_guard<std::mutex> l(g_tune_mu);
    return save_file_locked(path);
}

int b2co_tune_cache_load(char const* path)
{
    if (!path) return fail(B2CO_EINVAL, "null path");
    std::lock_guard<std::mutex> l(g_tune_mu);
    return load_file_locked(path);
}

int b2co_tune_cache_clear(void)
{
    std::lock_guard<std::mutex> l(g_tune_mu);
    g_tune.clear();
    return B2CO_OK;
}

}  // extern "C"
