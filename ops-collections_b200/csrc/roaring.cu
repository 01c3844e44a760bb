// roaring.cu -- RoaringBitmap<Key> (Key uint32 or uint64) over the portable
// Roaring serialization (RoaringFormatSpec), as in the reference
// (include/roaring_bitmap.h, detail/roaring_bitmap/format.h,
// roaring_bitmap_ref.h): the bytes are parsed and validated on the host, kept
// verbatim in device memory (Data()), and queried with Contains.
//
// B200 design: the host parse also flattens the container directory -- every
// container's high key (u16), kind, cardinality and byte offset, and for
// 64-bit keys every bucket's high key and container range -- into small device
// arrays.  For 32-bit keys a direct table maps each of the 65,536 high keys to
// its container (256 KiB, L2-resident), so a lookup is one table read plus one
// container probe; for 64-bit keys a query block stages the bucket and
// container keys in shared memory when they fit and binary-searches them.  The
// container probe reads the serialized bytes: an array (binary search of
// sorted u16), a bitset (one byte) or a run container (binary search of run
// starts).  Container data may sit at odd byte offsets; such containers are
// read byte-wise, the others with 16-bit loads.
#include <algorithm>
#include <limits>
#include <new>
#include <vector>

#include "b2co_host.h"

using namespace b2co;

namespace {

constexpr uint64_t kUnbounded = ~0ull;
constexpr uint32_t kCookieNoRun = 12346, kCookieRun = 12347;
constexpr uint32_t kMaxContainers = 1u << 16;
constexpr uint32_t kMaxArray = 4096;
constexpr uint32_t kBitsetBytes = 8192;
constexpr uint32_t kNoOffsetThreshold = 4;

enum : uint32_t { kArray = 0, kBitset = 1, kRun = 2, kKindMask = 0xff, kAligned = 0x100 };
constexpr uint32_t kNoContainer = 0xffffffffu;

struct alignas(16) Container {
    unsigned long long offset;  // bytes from the start of the serialized data
    uint32_t card;              // cardinality (array / bitset)
    uint32_t kind;
};

// ---- host parse ----------------------------------------------------------------

struct Reader {
    uint8_t const* p;
    uint64_t avail;  // kUnbounded: trust the format
    bool ok = true;
    bool require(uint64_t off, uint64_t n)
    {
        if (avail == kUnbounded) return true;
        if (off > avail || n > avail - off) ok = false;
        return ok;
    }
    uint32_t u16(uint64_t off) { return require(off, 2) ? uint32_t(p[off]) | (uint32_t(p[off + 1]) << 8) : 0; }
    uint32_t u32(uint64_t off) { return require(off, 4) ? u16(off) | (u16(off + 2) << 16) : 0; }
    uint64_t u64(uint64_t off) { return require(off, 8) ? uint64_t(u32(off)) | (uint64_t(u32(off + 4)) << 32) : 0; }
};

// Parses one 32-bit portable bitmap at `base` (offsets in the output are
// absolute, i.e. relative to the whole serialized buffer).  The checks follow
// ParseRoaringBitmap32 (format.h:164-262).
int parse32(uint8_t const* data, uint64_t avail, uint64_t base, std::vector<uint16_t>& keys,
            std::vector<Container>& out, uint64_t* num_keys, uint64_t* size_bytes)
{
    Reader r{data + base, avail};
    uint32_t const cookie = r.u32(0);
    if (!r.ok) return fail(B2CO_EINVAL, "RoaringBitmap: truncated serialized bitmap");
    uint64_t cursor = 4, run_bitmap = 0;
    uint32_t n = 0;
    bool has_run = false;
    if ((cookie & 0xffffu) == kCookieRun) {
        has_run = true;
        n = (cookie >> 16) + 1;
        run_bitmap = cursor;
        cursor += (uint64_t(n) + 7) / 8;
    } else if (cookie == kCookieNoRun) {
        n = r.u32(cursor);
        cursor += 4;
    } else {
        return fail(B2CO_EINVAL, "RoaringBitmap: unsupported serialized cookie");
    }
    if (!r.ok) return fail(B2CO_EINVAL, "RoaringBitmap: truncated serialized bitmap");
    if (n > kMaxContainers) return fail(B2CO_EINVAL, "RoaringBitmap: container count is out of range");
    if (has_run && !r.require(run_bitmap, (uint64_t(n) + 7) / 8))
        return fail(B2CO_EINVAL, "RoaringBitmap: truncated serialized bitmap");
    uint64_t const key_cards = cursor;
    if (!r.require(cursor, uint64_t(n) * 4)) return fail(B2CO_EINVAL, "RoaringBitmap: truncated serialized bitmap");
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t const k = r.u16(key_cards + 4ull * i);
        if (i && k <= keys.back()) return fail(B2CO_EINVAL, "RoaringBitmap: container keys must be strictly increasing");
        keys.push_back(uint16_t(k));
        total += uint64_t(r.u16(key_cards + 4ull * i + 2)) + 1;
    }
    cursor += uint64_t(n) * 4;
    bool const serialized_offsets = !has_run || n >= kNoOffsetThreshold;
    uint64_t const offsets_at = cursor;
    if (serialized_offsets) {
        if (!r.require(cursor, uint64_t(n) * 4)) return fail(B2CO_EINVAL, "RoaringBitmap: truncated serialized bitmap");
        cursor += uint64_t(n) * 4;
    }
    uint64_t prev_end = cursor;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t const card = r.u16(key_cards + 4ull * i + 2) + 1;
        uint64_t off = prev_end;
        if (serialized_offsets) {
            off = r.u32(offsets_at + 4ull * i);
            if (off < cursor || off < prev_end) return fail(B2CO_EINVAL, "RoaringBitmap: invalid container offset");
        }
        bool const is_run = has_run && ((r.p[run_bitmap + i / 8] >> (i % 8)) & 1u);
        uint64_t bytes;
        uint32_t kind;
        if (is_run) {
            bytes = 2 + 4ull * r.u16(off);
            kind = kRun;
        } else if (card <= kMaxArray) {
            bytes = 2ull * card;
            kind = kArray;
        } else {
            bytes = kBitsetBytes;
            kind = kBitset;
        }
        if (!r.require(off, bytes) || !r.ok) return fail(B2CO_EINVAL, "RoaringBitmap: truncated serialized bitmap");
        if (((base + off) & 1) == 0) kind |= kAligned;  // 16-bit fields can be loaded as u16
        out.push_back(Container{base + off, card, kind});
        prev_end = off + bytes;
    }
    *num_keys = total;
    *size_bytes = prev_end;
    return B2CO_OK;
}

struct Parsed {
    std::vector<uint16_t> ckeys;
    std::vector<Container> cont;
    std::vector<uint32_t> bkeys;    // 64-bit: bucket high keys
    std::vector<uint32_t> bstart;   // 64-bit: first container of each bucket (+ end)
    uint64_t num_keys = 0, size_bytes = 0;
};

int parse(uint8_t const* data, uint64_t avail, uint32_t key_bytes, Parsed& p)
{
    if (!data) return fail(B2CO_EINVAL, "RoaringBitmap: bitmap must not be null");
    if (key_bytes == 4) {
        return parse32(data, avail, 0, p.ckeys, p.cont, &p.num_keys, &p.size_bytes);
    }
    // 64-bit portable bucketed form (format.h:269-318)
    Reader r{data, avail};
    uint64_t const nb = r.u64(0);
    if (!r.ok) return fail(B2CO_EINVAL, "RoaringBitmap: truncated serialized bitmap");
    uint64_t cursor = 8;
    if (avail != kUnbounded && nb > (avail - cursor) / 12)
        return fail(B2CO_EINVAL, "RoaringBitmap: truncated 64-bit bucket table");
    if (nb > (1ull << 32)) return fail(B2CO_EINVAL, "RoaringBitmap: bucket count is out of range");
    for (uint64_t b = 0; b < nb; ++b) {
        uint32_t const k = r.u32(cursor);
        if (!r.ok) return fail(B2CO_EINVAL, "RoaringBitmap: truncated serialized bitmap");
        if (b && k <= p.bkeys.back()) return fail(B2CO_EINVAL, "RoaringBitmap: bucket keys must be strictly increasing");
        cursor += 4;
        p.bkeys.push_back(k);
        p.bstart.push_back(uint32_t(p.cont.size()));
        uint64_t const remaining = avail == kUnbounded ? kUnbounded : avail - cursor;
        std::vector<uint16_t> keys;
        uint64_t nk = 0, sb = 0;
        if (int st = parse32(data, remaining, cursor, keys, p.cont, &nk, &sb)) return st;
        p.ckeys.insert(p.ckeys.end(), keys.begin(), keys.end());
        p.num_keys += nk;
        cursor += sb;
    }
    p.bstart.push_back(uint32_t(p.cont.size()));
    p.size_bytes = cursor;
    return B2CO_OK;
}

// ---- device query ----------------------------------------------------------------

__device__ __forceinline__ uint32_t ld16(uint8_t const* p) { return uint32_t(__ldg(p)) | (uint32_t(__ldg(p + 1)) << 8); }

// First index in [lo, hi) whose key is >= k (keys in shared or global memory).
template <class T>
__device__ __forceinline__ uint32_t lower_bound(T const* keys, uint32_t lo, uint32_t hi, uint32_t k)
{
    while (lo < hi) {
        uint32_t const mid = (lo + hi) >> 1;
        if (uint32_t(keys[mid]) < k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool container_has(uint8_t const* bytes, Container const& c, uint32_t low)
{
    uint8_t const* p = bytes + c.offset;
    uint32_t const kind = c.kind & kKindMask;
    if (kind == kBitset) return (__ldg(p + (low >> 3)) >> (low & 7)) & 1u;
    if (kind == kArray) {
        uint32_t lo = 0, hi = c.card;
        uint16_t const* a = reinterpret_cast<uint16_t const*>(p);
        bool const aligned = c.kind & kAligned;
        while (lo < hi) {
            uint32_t const mid = (lo + hi) >> 1;
            uint32_t const v = aligned ? uint32_t(__ldg(a + mid)) : ld16(p + 2 * mid);
            if (v == low) return true;
            if (v < low) lo = mid + 1;
            else hi = mid;
        }
        return false;
    }
    // run container: the last run whose start <= low, then its end (start + length)
    uint32_t const runs = ld16(p);
    uint32_t lo = 0, hi = runs;
    while (lo < hi) {
        uint32_t const mid = (lo + hi) >> 1;
        if (ld16(p + 2 + 4 * mid) <= low) lo = mid + 1;
        else hi = mid;
    }
    if (lo == 0) return false;
    uint8_t const* run = p + 2 + 4 * (lo - 1);
    return low <= ld16(run) + ld16(run + 2);
}

constexpr uint32_t kSharedKeys = 16384;  // u16 container keys staged per block (32 KiB)
constexpr uint32_t kSharedBuckets = 2048;

// 32-bit keys: a direct table from the 16-bit high key to the container
// (65,536 entries, 256 KiB, L2-resident) replaces the directory search.
__global__ void __launch_bounds__(256) k_roaring_contains32(uint8_t const* bytes, uint32_t const* direct,
                                                            Container const* cont, uint32_t const* keys, uint8_t* out,
                                                            uint64_t n)
{
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t const key = __ldg(keys + i);
        uint32_t const c = __ldg(direct + (key >> 16));
        out[i] = c != kNoContainer && container_has(bytes, cont[c], key & 0xffffu);
    }
}

// 64-bit keys: bucket search, then the bucket's container directory, both on
// chip when they fit.
__global__ void __launch_bounds__(256) k_roaring_contains64(uint8_t const* bytes, uint16_t const* ckeys,
                                                            Container const* cont, uint32_t ncont,
                                                            uint32_t const* bkeys, uint32_t const* bstart,
                                                            uint32_t nbuckets, unsigned long long const* keys,
                                                            uint8_t* out, uint64_t n, bool stage)
{
    __shared__ uint16_t s_ckeys[kSharedKeys];
    __shared__ uint32_t s_bkeys[kSharedBuckets];
    if (stage) {
        for (uint32_t i = threadIdx.x; i < ncont; i += blockDim.x) s_ckeys[i] = ckeys[i];
        for (uint32_t i = threadIdx.x; i < nbuckets; i += blockDim.x) s_bkeys[i] = bkeys[i];
        __syncthreads();
    }
    uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint64_t const key = __ldg(keys + i);
        uint32_t const hk = uint32_t(key >> 32);
        uint32_t const b = stage ? lower_bound(s_bkeys, 0, nbuckets, hk) : lower_bound(bkeys, 0, nbuckets, hk);
        uint8_t r = 0;
        if (b < nbuckets && (stage ? s_bkeys[b] : bkeys[b]) == hk) {
            uint32_t const lo = bstart[b], hi = bstart[b + 1];
            uint32_t const ck = uint32_t(key >> 16) & 0xffffu;
            uint32_t const c = stage ? lower_bound(s_ckeys, lo, hi, ck) : lower_bound(ckeys, lo, hi, ck);
            if (c < hi && (stage ? uint32_t(s_ckeys[c]) : uint32_t(ckeys[c])) == ck)
                r = container_has(bytes, cont[c], uint32_t(key) & 0xffffu);
        }
        out[i] = r;
    }
}

cudaStream_t cs(b2co_stream s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

struct b2co_roaring {
    uint32_t key_bytes = 0;
    uint64_t num_keys = 0, size_bytes = 0;
    uint8_t* bytes = nullptr;  // the serialized bitmap (Data())
    uint16_t* ckeys = nullptr;
    Container* cont = nullptr;
    uint32_t* bkeys = nullptr;
    uint32_t* bstart = nullptr;
    uint32_t* direct = nullptr;  // 32-bit keys: high key -> container
    uint32_t ncont = 0, nbuckets = 0;
};

namespace {

int check(b2co_roaring const* r)
{
    if (!r) return fail(B2CO_ELOGIC, "RoaringBitmap: moved-from object");
    return B2CO_OK;
}

template <class T>
int upload(T** dst, std::vector<T> const& src, cudaStream_t s)
{
    size_t const bytes = std::max<size_t>(src.size(), 1) * sizeof(T);
    B2CO_CUDA(cudaMalloc(reinterpret_cast<void**>(dst), bytes));
    if (!src.empty()) B2CO_CUDA(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return B2CO_OK;
}

int contains_impl(b2co_roaring* r, void const* keys, uint8_t* out, uint64_t n, cudaStream_t s)
{
    if (int st = check(r)) return st;
    if (n == 0) return B2CO_OK;
    if (!keys || !out) return fail(B2CO_EINVAL, "RoaringBitmap: null input or output with a nonzero key count");
    if (n > kMaxBatch) return fail(B2CO_ERANGE, "RoaringBitmap: batch exceeds the 32-bit index range");
    if (r->key_bytes == 4) {
        auto k = k_roaring_contains32;
        k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(r->bytes, r->direct, r->cont,
                                                               static_cast<uint32_t const*>(keys), out, n);
    } else {
        bool const stage = r->ncont <= kSharedKeys && r->nbuckets <= kSharedBuckets;
        auto k = k_roaring_contains64;
        k<<<grid_for((void const*)k, 256, n, 256), 256, 0, s>>>(r->bytes, r->ckeys, r->cont, r->ncont, r->bkeys,
                                                               r->bstart, r->nbuckets,
                                                               static_cast<unsigned long long const*>(keys), out, n,
                                                               stage);
    }
    B2CO_CUDA(cudaGetLastError());
    return B2CO_OK;
}

}  // namespace

extern "C" {

int b2co_roaring_parse(void const* host_bytes, uint64_t available_bytes, uint32_t key_bytes, uint64_t* num_keys,
                       uint64_t* size_bytes)
{
    if (key_bytes != 4 && key_bytes != 8) return fail(B2CO_EINVAL, "RoaringBitmap: keys are 4 or 8 bytes");
    Parsed p;
    if (int st = parse(static_cast<uint8_t const*>(host_bytes), available_bytes, key_bytes, p)) return st;
    if (num_keys) *num_keys = p.num_keys;
    if (size_bytes) *size_bytes = p.size_bytes;
    return B2CO_OK;
}

int b2co_roaring_create(void const* host_bytes, uint64_t available_bytes, uint32_t key_bytes, b2co_stream stream,
                        b2co_roaring** out)
{
    if (!out) return fail(B2CO_EINVAL, "null output");
    *out = nullptr;
    if (key_bytes != 4 && key_bytes != 8) return fail(B2CO_EINVAL, "RoaringBitmap: keys are 4 or 8 bytes");
    Parsed p;
    if (int st = parse(static_cast<uint8_t const*>(host_bytes), available_bytes, key_bytes, p)) return st;
    auto* r = new (std::nothrow) b2co_roaring;
    if (!r) return fail(B2CO_ENOMEM, "host allocation failed");
    r->key_bytes = key_bytes;
    r->num_keys = p.num_keys;
    r->size_bytes = p.size_bytes;
    r->ncont = uint32_t(p.cont.size());
    r->nbuckets = uint32_t(p.bkeys.size());
    cudaStream_t s = cs(stream);
    std::vector<uint8_t> raw(static_cast<uint8_t const*>(host_bytes),
                             static_cast<uint8_t const*>(host_bytes) + p.size_bytes);
    int st = upload(&r->bytes, raw, s);
    if (!st) st = upload(&r->ckeys, p.ckeys, s);
    if (!st) st = upload(&r->cont, p.cont, s);
    if (!st) st = upload(&r->bkeys, p.bkeys, s);
    if (!st) st = upload(&r->bstart, p.bstart.empty() ? std::vector<uint32_t>{0u} : p.bstart, s);
    if (!st && key_bytes == 4) {
        std::vector<uint32_t> direct(1u << 16, kNoContainer);
        for (uint32_t c = 0; c < r->ncont; ++c) direct[p.ckeys[c]] = c;
        st = upload(&r->direct, direct, s);
        if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = cuda_fail(cudaGetLastError(), "RoaringBitmap upload");
    }
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = cuda_fail(cudaGetLastError(), "RoaringBitmap upload");
    if (st) {
        b2co_roaring_destroy(r);
        return st;
    }
    *out = r;
    return B2CO_OK;
}

int b2co_roaring_destroy(b2co_roaring* r)
{
    if (!r) return B2CO_OK;
    cudaFree(r->bytes);
    cudaFree(r->ckeys);
    cudaFree(r->cont);
    cudaFree(r->bkeys);
    cudaFree(r->bstart);
    cudaFree(r->direct);
    delete r;
    return B2CO_OK;
}

int b2co_roaring_contains_async(b2co_roaring* r, void const* keys, uint8_t* out, uint64_t n, b2co_stream s)
{
    return contains_impl(r, keys, out, n, cs(s));
}

int b2co_roaring_contains(b2co_roaring* r, void const* keys, uint8_t* out, uint64_t n, b2co_stream s)
{
    if (int st = contains_impl(r, keys, out, n, cs(s))) return st;
    B2CO_CUDA(cudaStreamSynchronize(cs(s)));
    return B2CO_OK;
}

int b2co_roaring_size(b2co_roaring const* r, uint64_t* num_keys)
{
    if (int st = check(r)) return st;
    if (!num_keys) return fail(B2CO_EINVAL, "null output");
    *num_keys = r->num_keys;
    return B2CO_OK;
}

int b2co_roaring_size_bytes(b2co_roaring const* r, uint64_t* size_bytes)
{
    if (int st = check(r)) return st;
    if (!size_bytes) return fail(B2CO_EINVAL, "null output");
    *size_bytes = r->size_bytes;
    return B2CO_OK;
}

int b2co_roaring_data(b2co_roaring const* r, uint8_t const** device_bytes)
{
    if (int st = check(r)) return st;
    if (!device_bytes) return fail(B2CO_EINVAL, "null output");
    *device_bytes = r->bytes;
    return B2CO_OK;
}

}  // extern "C"
