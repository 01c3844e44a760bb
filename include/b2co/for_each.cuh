// for_each.cuh -- ForEach / ForEachAsync over a StaticMap or StaticSet with a
// caller-defined device functor, compiled by the caller's nvcc (a functor
// cannot cross the library's C ABI).  Include <b2co/b2co.hpp> from a .cu file:
// it pulls this header in and adds the ForEach member templates.
//
// Semantics follow the reference (detail/open_addressing/open_addressing_ref_impl.h:
// 424-454 ForEach, kernels.h:379-406 ForEachSimt, open_addressing_impl.h:325-339
// ForEachAsync): for every probe key, walk its probe sequence bucket by bucket;
// a slot whose key is bitwise the empty key ends the walk, a slot whose key
// equals the probe key (operator==) is handed to the callback as its Pair
// (StaticMap) or key (StaticSet), and the walk ends after a full cycle.  The
// callback type is constructed on the device from the `callbackArgs` pointer
// (CallbackOp(uint8_t*)), like the reference's `__gm__ uint8_t*` constructor,
// and must not modify the table.
#pragma once

#include "b2co.hpp"
#include "device.cuh"

namespace b2co {
namespace detail {

inline void cuda_check(cudaError_t e, char const* what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
__device__ __forceinline__ T from_bits(uint64_t b)
{
    T v;
    memcpy(&v, &b, sizeof(T));
    return v;
}

template <class CallbackOp, class Key, class T, int B>
__global__ void __launch_bounds__(256) k_for_each(void const* slots, ProbeParams p, uint64_t empty_key,
                                                 Key const* keys, uint32_t n, uint8_t* callback_args)
{
    constexpr bool kSet = std::is_void<T>::value;
    using S = SlotT<int(sizeof(Key)), kSet ? 0 : int(sizeof(typename std::conditional<kSet, int, T>::type))>;
    using Raw = typename S::Raw;
    Raw const* table = static_cast<Raw const*>(slots);
    CallbackOp callback(callback_args);
    uint32_t const stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Key const key = keys[i];
        uint64_t kb = 0;
        memcpy(&kb, &key, sizeof(Key));
        uint32_t idx = probe_init<int(sizeof(Key)), B>(p, kb);
        uint32_t const step = probe_step<int(sizeof(Key)), B>(p, kb);
        uint32_t const init = idx;
        bool done = false;
        while (!done) {
#pragma unroll
            for (int j = 0; j < B; ++j) {
                Raw const r = table[idx + j];
                uint64_t const sk = S::key(r);
                if (sk == empty_key) {
                    done = true;
                    break;
                }
                if (from_bits<Key>(sk) == key) {
                    if constexpr (kSet) {
                        callback(from_bits<Key>(sk));
                    } else {
                        Pair<Key, T> pr;
                        pr.first = from_bits<Key>(sk);
                        pr.second = from_bits<T>(S::value(r));
                        callback(pr);
                    }
                }
            }
            if (done) break;
            idx = probe_next(idx, step, p.capacity);
            done = idx == init;
        }
    }
}

template <class CallbackOp, class Key, class T, int B>
void launch_for_each(b2co_oa_desc const& d, void const* slots, uint64_t capacity, void* keys, uint32_t n,
                     void* args, cudaStream_t stream)
{
    ProbeParams const p = make_probe_params(capacity, B, d.probing, d.hash);
    int dev = 0, sms = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    uint64_t const want = (uint64_t(n) + 255) / 256, most = uint64_t(sms) * 8;
    uint32_t const blocks = uint32_t(want < most ? want : most);
    k_for_each<CallbackOp, Key, T, B><<<blocks, 256, 0, stream>>>(slots, p, d.empty_key_bits, static_cast<Key const*>(keys),
                                                                   n, static_cast<uint8_t*>(args));
    cuda_check(cudaGetLastError(), "ForEach launch");
}

// The kernels index in uint32 like every other batch call (open_addressing_impl.h:534-545).
constexpr uint64_t kForEachMaxBatch = 0xFFFFFFFFull - (1ull << 22);

template <class CallbackOp, class Key, class T>
void for_each_async(b2co_oa_table* t, void* keys, uint64_t n, void* args, cudaStream_t stream)
{
    if (n == 0 || keys == nullptr) return;
    if (n > kForEachMaxBatch) throw std::length_error("ForEach batch exceeds the 32-bit index range");
    b2co_oa_desc d{};
    throw_on(b2co_oa_describe(t, &d));
    void* slots = nullptr;
    throw_on(b2co_oa_data(t, &slots));
    uint64_t cap = 0;
    throw_on(b2co_oa_capacity(t, &cap));
    uint32_t const m = uint32_t(n);
    switch (d.bucket_size) {
        case 1: return launch_for_each<CallbackOp, Key, T, 1>(d, slots, cap, keys, m, args, stream);
        case 2: return launch_for_each<CallbackOp, Key, T, 2>(d, slots, cap, keys, m, args, stream);
        case 4: return launch_for_each<CallbackOp, Key, T, 4>(d, slots, cap, keys, m, args, stream);
        case 5: return launch_for_each<CallbackOp, Key, T, 5>(d, slots, cap, keys, m, args, stream);
        case 8: return launch_for_each<CallbackOp, Key, T, 8>(d, slots, cap, keys, m, args, stream);
        default: throw std::invalid_argument("ForEach: unsupported bucket size");
    }
}

}  // namespace detail
}  // namespace b2co
