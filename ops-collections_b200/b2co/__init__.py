"""Python host layer over libb2co.so, mirroring the reference's container API.

The reference (ops-collections) exposes C++ class templates -- StaticMap,
StaticSet, DynamicMap, BloomFilter, HyperLogLog -- whose methods take device
pointers, a count and a stream.  These classes keep the same method names,
argument meaning and error behaviour, over the C ABI declared in
include/b2co.h.  Device buffers are torch CUDA tensors (plumbing only); every
operation runs in libb2co's own sm_100a kernels.  There is no CPU fallback:
without the built library every call raises.

Exceptions map the reference's C++ exceptions:
    std::invalid_argument -> InvalidArgument (ValueError)
    std::length_error     -> LengthError (ValueError)
    std::bad_alloc        -> BadAlloc (MemoryError)
    std::runtime_error    -> CudaError (RuntimeError)
    std::logic_error      -> LogicError (RuntimeError)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# B2CO_LIB names another build of the same library (e.g. one compiled with other tuning macros).
LIB_PATH = os.environ.get("B2CO_LIB") or os.path.join(os.path.dirname(_HERE), "lib", "libb2co.so")

OK, EINVAL, ERANGE, ENOMEM, ECUDA, ETIMEOUT, ELOGIC, EOVERFLOW = range(8)
HASH_XXH32, HASH_MURMUR3_32, HASH_FMIX, HASH_XXH64 = range(4)
PROBE_LINEAR, PROBE_DOUBLE = 0, 1
IAF_RACE, IAF_FIRST_WINS = 0, 1
INSERT_EXACT_DEDUP, INSERT_APPEND_UNIQUE = 0, 1
FIND_SEGMENTED = 0x100
FIND_BULK = 0x200
FIND_WARP_STAGED = 0x400
FIND_DEFERRED = 0x800
BLOOM_ADD_ATOMIC, BLOOM_ADD_BULK, BLOOM_ADD_PARTITIONED, BLOOM_ADD_AUTO = 0, 1, 2, 3


class B2coError(Exception):
    status = -1


class InvalidArgument(B2coError, ValueError):
    status = EINVAL


class LengthError(B2coError, ValueError):
    status = ERANGE


class BadAlloc(B2coError, MemoryError):
    status = ENOMEM


class CudaError(B2coError, RuntimeError):
    status = ECUDA


class TimeoutError_(B2coError, RuntimeError):
    status = ETIMEOUT


class LogicError(B2coError, RuntimeError):
    status = ELOGIC


class OverflowError_(B2coError, OverflowError):
    status = EOVERFLOW


_EXC = {EINVAL: InvalidArgument, ERANGE: LengthError, ENOMEM: BadAlloc, ECUDA: CudaError,
        ETIMEOUT: TimeoutError_, ELOGIC: LogicError, EOVERFLOW: OverflowError_}


class OaDesc(C.Structure):
    _fields_ = [("key_bytes", C.c_uint32), ("value_bytes", C.c_uint32), ("bucket_size", C.c_uint32),
                ("probing", C.c_uint32), ("hash", C.c_uint32), ("key_kind", C.c_uint32),
                ("empty_key_bits", C.c_uint64), ("empty_value_bits", C.c_uint64),
                ("erased_key_bits", C.c_uint64)]


_lib = None


def lib():
    """The loaded libb2co.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libb2co.so is not built ({LIB_PATH}); run ops-collections_b200/build.py")
        L = C.CDLL(LIB_PATH)
        L.b2co_last_error.restype = C.c_char_p
        L.b2co_status_string.restype = C.c_char_p
        L.b2co_version.restype = C.c_char_p
        L.b2co_server_now_ns.restype = C.c_uint64
        _lib = L
    return _lib


def _check(status: int):
    if status != OK:
        msg = lib().b2co_last_error().decode(errors="replace")
        raise _EXC.get(status, B2coError)(msg or lib().b2co_status_string(status).decode())


def _call(name, *args):
    _check(getattr(lib(), name)(*args))


def _ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    """A cudaStream_t handle: a torch.cuda.Stream, a raw int handle, or None for torch's current stream."""
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


KEY_INTEGER, KEY_FLOAT = 0, 1
_FLOATS = {2: np.float16, 4: np.float32, 8: np.float64}
_UINTS = {2: np.uint16, 4: np.uint32, 8: np.uint64}


def _bits(x, nbytes: int, floating: bool = False) -> int:
    """Bit pattern of a sentinel: the IEEE encoding of that width for a float
    (or for any value when `floating`), two's complement for an integer."""
    if floating or isinstance(x, (float, np.floating)):
        return int(np.array([x], dtype=_FLOATS[nbytes]).view(_UINTS[nbytes])[0])
    return int(x) & ((1 << (8 * nbytes)) - 1)


def _is_float(dt) -> bool:
    return dt is not None and dt.is_floating_point


def slot_bytes(key_bytes: int, value_bytes: int) -> int:
    """Pair<K,V> aligned to min(16, bitceil(sizeof K + sizeof V)), payload at the
    next offset aligned to its own size (pair.inl:19-24); a set slot is the key."""
    if value_bytes == 0:
        return key_bytes
    s = key_bytes + value_bytes
    align = 4 if s <= 4 else (8 if s <= 8 else 16)
    end = (key_bytes + value_bytes - 1) // value_bytes * value_bytes + value_bytes
    return (end + align - 1) // align * align


def pack_pairs(keys, values):
    """Device array of Pair<K,V> slots (the reference's `values` argument) from key and payload tensors."""
    import torch
    kb, vb = keys.element_size(), values.element_size()
    n = keys.numel()
    if kb == 4 and vb == 4:
        return torch.stack([keys.view(torch.int32), values.view(torch.int32)], dim=1).contiguous()
    if kb == 2 and vb == 2:
        return torch.stack([keys.view(torch.int16), values.view(torch.int16)], dim=1).contiguous()
    out = torch.zeros((n, 2), dtype=torch.int64, device=keys.device)
    if kb == 8:
        out[:, 0] = keys.view(torch.int64)
    else:
        out[:, 0] = keys.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    if vb == 8:
        out[:, 1] = values.view(torch.int64)
    else:
        out[:, 1] = values.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    return out


def _int_view(t):
    """The tensor's bits as a signed integer tensor of the same width."""
    import torch
    return t.view({2: torch.int16, 4: torch.int32, 8: torch.int64}[t.element_size()])


def set_l2_fetch_granularity(nbytes: int) -> int:
    """Context-wide hint of how many bytes the L2 fetches from DRAM per miss
    (32, 64 or 128).  Random bucket windows waste most of a 128-byte line; a
    smaller granularity cuts DRAM traffic per lookup.  Applies to the whole
    process's CUDA context, so it is the application's choice to make."""
    v = C.c_uint64()
    _call("b2co_set_l2_fetch_granularity", C.c_uint32(nbytes), C.byref(v))
    return v.value


def valid_capacity(requested: int, bucket_size: int = 5, probing: int = PROBE_DOUBLE) -> int:
    c = C.c_uint64()
    _call("b2co_oa_valid_capacity", C.c_uint64(requested), C.c_uint32(bucket_size), C.c_uint32(probing),
          C.byref(c))
    return c.value


def _dtype_bytes(dt) -> int:
    import torch
    return torch.empty((), dtype=dt).element_size()


class _OaBase:
    """Shared implementation of StaticMap and StaticSet (OpenAddressingImpl)."""

    def __init__(self, capacity, empty_key, empty_value, key_dtype, value_dtype, bucket_size, probing, hash_kind,
                 erased_key, stream):
        import torch
        self.key_dtype = key_dtype
        self.value_dtype = value_dtype
        kb = _dtype_bytes(key_dtype)
        vb = 0 if value_dtype is None else _dtype_bytes(value_dtype)
        self.key_bytes, self.value_bytes = kb, vb
        self.empty_key, self.empty_value = empty_key, empty_value
        fk, fv = _is_float(key_dtype), _is_float(value_dtype)
        d = OaDesc(kb, vb, bucket_size, probing, hash_kind, KEY_FLOAT if fk else KEY_INTEGER, _bits(empty_key, kb, fk),
                   _bits(empty_value, vb, fv) if vb else 0,
                   _bits(empty_key if erased_key is None else erased_key, kb, fk))
        self._desc = d
        h = C.c_void_p()
        _call("b2co_oa_create", C.byref(d), C.c_uint64(capacity), _stream(stream), C.byref(h))
        self._h = h
        self.bucket_size = bucket_size

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.b2co_oa_destroy(h)
            self._h = None

    # -- properties (static_map.h:584, :604) ---------------------------------
    def Capacity(self) -> int:
        c = C.c_uint64()
        _call("b2co_oa_capacity", self._h, C.byref(c))
        return c.value

    def Data(self) -> int:
        p = C.c_void_p()
        _call("b2co_oa_data", self._h, C.byref(p))
        return p.value

    def slot_bytes(self) -> int:
        return slot_bytes(self.key_bytes, self.value_bytes)

    def dump_slots(self) -> np.ndarray:
        """Raw slot bytes copied to the host (numpy uint8, capacity * slot_bytes)."""
        return _device_bytes(self.Data(), self.Capacity() * self.slot_bytes())

    def SetErasedKey(self, erased_key, stream=None):
        _call("b2co_oa_set_erased_key", self._h,
              C.c_uint64(_bits(erased_key, self.key_bytes, _is_float(self.key_dtype))), _stream(stream))

    def Clear(self, stream=None):
        _call("b2co_oa_clear", self._h, _stream(stream))

    def ClearAsync(self, stream=None):
        _call("b2co_oa_clear_async", self._h, _stream(stream))

    # -- inserts --------------------------------------------------------------
    def Insert(self, values, n=None, stream=None) -> int:
        f = C.c_uint64()
        _call("b2co_oa_insert", self._h, _ptr(values), C.c_uint64(self._n(values, n)), _stream(stream),
              C.byref(f))
        return f.value

    def InsertAsync(self, values, n=None, stream=None):
        _call("b2co_oa_insert_async", self._h, _ptr(values), C.c_uint64(self._n(values, n)), _stream(stream))

    def InsertIf(self, values, stencil, n=None, stream=None) -> int:
        f = C.c_uint64()
        _call("b2co_oa_insert_if", self._h, _ptr(values), _ptr(stencil), C.c_uint64(self._n(values, n)),
              _stream(stream), C.byref(f))
        return f.value

    def InsertIfAsync(self, values, stencil, n=None, stream=None):
        _call("b2co_oa_insert_if_async", self._h, _ptr(values), _ptr(stencil), C.c_uint64(self._n(values, n)),
              _stream(stream))

    def InsertAndFind(self, values, output_find, output_insert, n=None, stream=None, mode=IAF_RACE):
        _call("b2co_oa_insert_and_find", self._h, _ptr(values), _ptr(output_find), _ptr(output_insert),
              C.c_uint64(self._n(values, n)), C.c_int(mode), _stream(stream))

    def InsertAndFindAsync(self, values, output_find, output_insert, n=None, stream=None, mode=IAF_RACE):
        _call("b2co_oa_insert_and_find_async", self._h, _ptr(values), _ptr(output_find), _ptr(output_insert),
              C.c_uint64(self._n(values, n)), C.c_int(mode), _stream(stream))

    def Erase(self, keys, n=None, stream=None) -> int:
        f = C.c_uint64()
        _call("b2co_oa_erase", self._h, _ptr(keys), C.c_uint64(self._n(keys, n)), _stream(stream), C.byref(f))
        return f.value

    def EraseAsync(self, keys, n=None, stream=None):
        _call("b2co_oa_erase_async", self._h, _ptr(keys), C.c_uint64(self._n(keys, n)), _stream(stream))

    # -- lookups ----------------------------------------------------------------
    def Find(self, keys, output_values, n=None, stream=None):
        _call("b2co_oa_find", self._h, _ptr(keys), _ptr(output_values), C.c_uint64(self._n(keys, n)),
              _stream(stream))

    def FindAsync(self, keys, output_values, n=None, stream=None):
        _call("b2co_oa_find_async", self._h, _ptr(keys), _ptr(output_values), C.c_uint64(self._n(keys, n)),
              _stream(stream))

    def FindIf(self, keys, stencil, output_values, n=None, stream=None):
        _call("b2co_oa_find_if", self._h, _ptr(keys), _ptr(stencil), _ptr(output_values),
              C.c_uint64(self._n(keys, n)), _stream(stream))

    def FindIfAsync(self, keys, stencil, output_values, n=None, stream=None):
        _call("b2co_oa_find_if_async", self._h, _ptr(keys), _ptr(stencil), _ptr(output_values),
              C.c_uint64(self._n(keys, n)), _stream(stream))

    def Contains(self, keys, output_values, n=None, stream=None):
        _call("b2co_oa_contains", self._h, _ptr(keys), _ptr(output_values), C.c_uint64(self._n(keys, n)),
              _stream(stream))

    def ContainsAsync(self, keys, output_values, n=None, stream=None):
        _call("b2co_oa_contains_async", self._h, _ptr(keys), _ptr(output_values), C.c_uint64(self._n(keys, n)),
              _stream(stream))

    def ContainsIf(self, keys, stencil, output_values, n=None, stream=None):
        _call("b2co_oa_contains_if", self._h, _ptr(keys), _ptr(stencil), _ptr(output_values),
              C.c_uint64(self._n(keys, n)), _stream(stream))

    def ContainsIfAsync(self, keys, stencil, output_values, n=None, stream=None):
        _call("b2co_oa_contains_if_async", self._h, _ptr(keys), _ptr(stencil), _ptr(output_values),
              C.c_uint64(self._n(keys, n)), _stream(stream))

    def Count(self, keys, n=None, stream=None) -> int:
        c = C.c_uint64()
        _call("b2co_oa_count", self._h, _ptr(keys), C.c_uint64(self._n(keys, n)), _stream(stream), C.byref(c))
        return c.value

    def FindHost(self, host_keys: np.ndarray, host_out: np.ndarray, stream=None):
        """Find with host (ideally pinned) buffers; copies overlap the probing."""
        n = len(host_keys)
        _call("b2co_oa_find_host", self._h, C.c_void_p(host_keys.ctypes.data), C.c_void_p(host_out.ctypes.data),
              C.c_uint64(n), _stream(stream))

    def window_gather(self, n: int, seed: int = 0, stream=None):
        """Bare random bucket-window reads over this table's slots (16- or 8-byte slots; a measurement aid)."""
        _call("b2co_oa_window_gather", self._h, C.c_uint64(n), C.c_uint32(seed), _stream(stream))

    def set_find_shape(self, lanes_per_key: int, keys_per_lane: int, segmented: bool = False, bulk: bool = False,
                       warp_staged: bool = False, deferred: bool = False):
        flags = (FIND_SEGMENTED if segmented else 0) | (FIND_BULK if bulk else 0) | \
            (FIND_WARP_STAGED if warp_staged else 0) | (FIND_DEFERRED if deferred else 0)
        _call("b2co_oa_set_find_shape", self._h, C.c_uint32(lanes_per_key), C.c_uint32(keys_per_lane | flags))

    def ReserveInsertAndFind(self, n: int):
        """Size first-wins InsertAndFind's scratch for batches up to n now (b2co_oa_reserve_insert_and_find)."""
        _call("b2co_oa_reserve_insert_and_find", self._h, C.c_uint64(n))

    def set_write_shape(self, lanes_per_key: int, keys_per_tile: int):
        """Kernel shape of the insert family (b2co_oa_set_write_shape); (0, 0) = default."""
        _call("b2co_oa_set_write_shape", self._h, C.c_uint32(lanes_per_key), C.c_uint32(keys_per_tile))

    @staticmethod
    def _n(t, n):
        if n is not None:
            return int(n)
        return 0 if t is None else int(t.shape[0])


def _device_bytes(ptr: int, nbytes: int) -> np.ndarray:
    """Copy `nbytes` of device memory at `ptr` into a host numpy array."""
    from cuda.bindings import runtime as rt
    out = np.empty(nbytes, dtype=np.uint8)
    (err,) = rt.cudaMemcpy(out.ctypes.data, ptr, nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    if err != rt.cudaError_t.cudaSuccess:
        raise CudaError(f"cudaMemcpy failed ({err})")
    return out


class StaticMap(_OaBase):
    """StaticMap<Key, T> (include/static_map.h:29-35).  Defaults follow the
    reference: LinearProbing<murmurhash3_32> with bucket size 5."""

    def __init__(self, capacity, empty_key, empty_value, key_dtype=None, value_dtype=None, bucket_size=5,
                 probing=PROBE_LINEAR, hash_kind=HASH_MURMUR3_32, erased_key=None, stream=None):
        import torch
        super().__init__(capacity, empty_key, empty_value, key_dtype or torch.int32, value_dtype or torch.int32,
                         bucket_size, probing, hash_kind, erased_key, stream)

    def InsertOrAssign(self, values, n=None, stream=None, with_assigned=False):
        f, a = C.c_uint64(), C.c_uint64()
        _call("b2co_oa_insert_or_assign", self._h, _ptr(values), C.c_uint64(self._n(values, n)), _stream(stream),
              C.byref(f), C.byref(a))
        return (f.value, a.value) if with_assigned else f.value

    def InsertOrAssignAsync(self, values, n=None, stream=None):
        _call("b2co_oa_insert_or_assign_async", self._h, _ptr(values), C.c_uint64(self._n(values, n)),
              _stream(stream))

    def AssignIfAsync(self, values, stencil, n=None, stream=None):
        _call("b2co_oa_assign_if_async", self._h, _ptr(values), _ptr(stencil), C.c_uint64(self._n(values, n)),
              _stream(stream))


class StaticSet(_OaBase):
    """StaticSet<Key> (include/static_set.h:27-32).  Defaults follow the
    reference: DoubleHashing<xxhash_32> with bucket size 5."""

    def __init__(self, capacity, empty_key, key_dtype=None, bucket_size=5, probing=PROBE_DOUBLE,
                 hash_kind=HASH_XXH32, erased_key=None, stream=None):
        import torch
        super().__init__(capacity, empty_key, 0, key_dtype or torch.int32, None, bucket_size, probing, hash_kind,
                         erased_key, stream)


class TableGroup:
    """Many independent StaticMap/StaticSet tables served by one launch per
    operation (include/b2co.h, b2co_oa_group_*).  `capacities` are the
    requested capacities per table; items of table t are the slice
    [offsets[t], offsets[t+1]) of a concatenated input."""

    def __init__(self, capacities, empty_key, empty_value, key_dtype=None, value_dtype=None, bucket_size=5,
                 probing=PROBE_DOUBLE, hash_kind=HASH_XXH32, stream=None):
        import torch
        key_dtype = key_dtype or torch.int32
        kb = _dtype_bytes(key_dtype)
        vb = 0 if value_dtype is None else _dtype_bytes(value_dtype)
        self.key_bytes, self.value_bytes = kb, vb
        caps = np.ascontiguousarray(capacities, dtype=np.uint64)
        d = OaDesc(kb, vb, bucket_size, probing, hash_kind, 0, _bits(empty_key, kb),
                   _bits(empty_value, vb) if vb else 0, _bits(empty_key, kb))
        h = C.c_void_p()
        _call("b2co_oa_group_create", C.byref(d), C.c_void_p(caps.ctypes.data), C.c_uint32(len(caps)),
              _stream(stream), C.byref(h))
        self._h = h
        self.count = len(caps)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.b2co_oa_group_destroy(h)
            self._h = None

    def table_capacity(self, t):
        v = C.c_uint64()
        _call("b2co_oa_group_table_capacity", self._h, C.c_uint32(t), C.byref(v))
        return v.value

    def total_slots(self):
        v = C.c_uint64()
        _call("b2co_oa_group_total_slots", self._h, C.byref(v))
        return v.value

    def Data(self) -> int:
        p = C.c_void_p()
        _call("b2co_oa_group_data", self._h, C.byref(p))
        return p.value

    def dump_slots(self) -> np.ndarray:
        return _device_bytes(self.Data(), self.total_slots() * slot_bytes(self.key_bytes, self.value_bytes))

    def Clear(self, stream=None):
        _call("b2co_oa_group_clear", self._h, _stream(stream))

    def Insert(self, pairs, d_offsets, stream=None, sync=True):
        f = C.c_uint64()
        _call("b2co_oa_group_insert", self._h, _ptr(pairs), _ptr(d_offsets), C.c_uint64(pairs.shape[0]),
              _stream(stream), C.byref(f) if sync else None)
        return f.value if sync else None

    def Find(self, keys, d_offsets, out, contains=False, stream=None, graph=False):
        name = "b2co_oa_group_find_graph" if graph else "b2co_oa_group_find"
        _call(name, self._h, _ptr(keys), _ptr(d_offsets), _ptr(out), C.c_uint64(keys.shape[0]),
              C.c_int(1 if contains else 0), _stream(stream))

    def FindPerTable(self, keys, h_offsets: np.ndarray, out, contains=False, stream=None):
        h = np.ascontiguousarray(h_offsets, dtype=np.uint64)
        _call("b2co_oa_group_find_per_table", self._h, _ptr(keys), C.c_void_p(h.ctypes.data), _ptr(out),
              C.c_int(1 if contains else 0), _stream(stream))

    def InsertPerTable(self, pairs, h_offsets: np.ndarray, stream=None):
        h = np.ascontiguousarray(h_offsets, dtype=np.uint64)
        _call("b2co_oa_group_insert_per_table", self._h, _ptr(pairs), C.c_void_p(h.ctypes.data), _stream(stream))

    def set_find_shape(self, lanes, keys_per_tile=1, block=0):
        _call("b2co_oa_group_set_find_shape_ex", self._h, C.c_uint32(lanes), C.c_uint32(keys_per_tile),
              C.c_uint32(block))

    def find_shape(self):
        """(lanes, keys per lane group, threads per block) of the group Find."""
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _call("b2co_oa_group_get_find_shape", self._h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def Autotune(self, keys, d_offsets, out, stream=None):
        """Times every group Find shape on this batch (or reuses the cached
        choice); returns ((lanes, keys per lane group, block), from_cache)."""
        a, b, c, hit = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_int()
        _call("b2co_oa_group_autotune", self._h, _ptr(keys), _ptr(d_offsets), _ptr(out), C.c_uint64(keys.shape[0]),
              _stream(stream), C.byref(a), C.byref(b), C.byref(c), C.byref(hit))
        return (a.value, b.value, c.value), bool(hit.value)


OP_FIND, OP_CONTAINS, OP_INSERT, OP_INSERT_OR_ASSIGN = 0, 1, 2, 3


class RequestInfo(C.Structure):
    _fields_ = [("id", C.c_uint64), ("op", C.c_int32), ("status", C.c_int32), ("n", C.c_uint64),
                ("arrival_ns", C.c_uint64), ("admit_ns", C.c_uint64), ("done_ns", C.c_uint64),
                ("failed", C.c_uint64), ("assigned", C.c_uint64)]


# numpy layouts of b2co_request_desc / b2co_request_info (batched submit / wait)
REQUEST_DESC = np.dtype([("table", "u8"), ("op", "i4"), ("reserved", "i4"), ("host_in", "u8"), ("host_out", "u8"),
                         ("n", "u8"), ("arrival_ns", "u8")])
REQUEST_INFO = np.dtype([("id", "u8"), ("op", "i4"), ("status", "i4"), ("n", "u8"), ("arrival_ns", "u8"),
                         ("admit_ns", "u8"), ("done_ns", "u8"), ("failed", "u8"), ("assigned", "u8")])


class Server:
    """Request server over resident tables (include/b2co.h, b2co_server_*).
    Host buffers passed to submit() must stay alive (and should be pinned)
    until the request completes."""

    _STATS_EX = ("launches", "requests_launched", "bytes_in_use", "staging_bytes", "staging_grows",
                 "max_launch_host_ns", "max_reserve_host_ns", "max_loop_gap_ns", "total_launch_host_ns", "copies",
                 "packed_launches", "direct_launches")

    def __init__(self, max_inflight=8, hbm_budget_bytes=150 << 30, max_batch_keys=0):
        L = lib()
        L.b2co_server_submit.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64,
                                         C.c_uint64, C.POINTER(C.c_uint64)]
        L.b2co_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(RequestInfo)]
        L.b2co_server_submit_many.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
        L.b2co_server_wait_many.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
        h = C.c_void_p()
        _call("b2co_server_create", C.c_uint32(max_inflight), C.c_uint64(hbm_budget_bytes),
              C.c_uint64(max_batch_keys), C.byref(h))
        self._h = h
        self._keep = {}
        self._rid = C.c_uint64()

    @staticmethod
    def now_ns() -> int:
        """The server clock (steady, ns) that arrival times are given in."""
        return lib().b2co_server_now_ns()

    def register(self, table):
        _call("b2co_server_register_table", self._h, table._h)

    def set_packing(self, on: bool):
        """Packed copies of coalesced launches (off by default)."""
        _call("b2co_server_set_packing", self._h, C.c_int(1 if on else 0))

    def set_direct_results(self, on: bool):
        """Lookup results written by the GPU into pinned host buffers (off by default)."""
        _call("b2co_server_set_direct_results", self._h, C.c_int(1 if on else 0))

    def set_plain(self, plain: bool):
        """Plain mode: one launch per request, one request per table at a time (the baseline)."""
        _call("b2co_server_set_plain", self._h, C.c_int(1 if plain else 0))

    def submit(self, table, op, host_in: np.ndarray, host_out=None, arrival_ns: int = 0) -> int:
        """Queues a request; the arrays are kept alive until wait() returns."""
        rid = self.submit_ptr(table._h.value, op, host_in.ctypes.data,
                              None if host_out is None else host_out.ctypes.data, host_in.shape[0], arrival_ns)
        self._keep[rid] = (host_in, host_out)
        return rid

    def submit_ptr(self, table_handle: int, op: int, in_ptr: int, out_ptr, n: int, arrival_ns: int = 0) -> int:
        """submit() on raw host addresses; the caller keeps the buffers alive."""
        st = _lib.b2co_server_submit(self._h, table_handle, op, in_ptr, out_ptr, n, arrival_ns, self._rid)
        if st != OK:
            _check(st)
        return self._rid.value

    def wait(self, rid: int) -> RequestInfo:
        info = RequestInfo()
        st = _lib.b2co_server_wait(self._h, rid, info)
        self._keep.pop(rid, None)
        if st != OK:
            _check(st)
        return info

    def submit_many(self, descs: np.ndarray) -> np.ndarray:
        """Submits a REQUEST_DESC array (table = a table's handle value, host
        addresses as integers) in one call; the caller keeps the buffers alive.
        Returns the ids."""
        descs = np.ascontiguousarray(descs, dtype=REQUEST_DESC)
        ids = np.empty(len(descs), dtype=np.uint64)
        st = _lib.b2co_server_submit_many(self._h, len(descs), descs.ctypes.data, ids.ctypes.data)
        if st != OK:
            _check(st)
        return ids

    def wait_many(self, ids, check: bool = True) -> np.ndarray:
        """Waits for every id; a REQUEST_INFO array.  With check, raises the
        first failed request's error after all have been waited for."""
        ids = np.ascontiguousarray(ids, dtype=np.uint64)
        infos = np.zeros(len(ids), dtype=REQUEST_INFO)
        st = _lib.b2co_server_wait_many(self._h, len(ids), ids.ctypes.data, infos.ctypes.data)
        for rid in ids.tolist():
            self._keep.pop(rid, None)
        if st != OK and check:
            _check(st)
        return infos

    def stats(self):
        """b2co_server_get_stats_ex as a dict."""
        v = (C.c_uint64 * len(self._STATS_EX))()
        _call("b2co_server_get_stats_ex", self._h, v)
        return dict(zip(self._STATS_EX, list(v)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value and _lib is not None:
            _lib.b2co_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def pinned(shape, dtype):
    """A numpy array in pinned (page-locked) host memory."""
    import torch
    tdt = {np.dtype(np.int64): torch.int64, np.dtype(np.int32): torch.int32, np.dtype(np.uint8): torch.uint8}[
        np.dtype(dtype)]
    return torch.empty(shape, dtype=tdt).pin_memory().numpy()


class DynamicMap:
    """DynamicMap<Key, T> (include/dynamic_map.h:26-29)."""

    kExactDedup, kAppendUnique = INSERT_EXACT_DEDUP, INSERT_APPEND_UNIQUE

    def __init__(self, initial_capacity, empty_key, empty_value, erased_key, key_dtype=None, value_dtype=None,
                 bucket_size=5, probing=PROBE_LINEAR, hash_kind=HASH_MURMUR3_32, stream=None):
        import torch
        key_dtype = key_dtype or torch.int32
        value_dtype = value_dtype or torch.int32
        kb, vb = _dtype_bytes(key_dtype), _dtype_bytes(value_dtype)
        self.key_bytes, self.value_bytes = kb, vb
        fk, fv = _is_float(key_dtype), _is_float(value_dtype)
        d = OaDesc(kb, vb, bucket_size, probing, hash_kind, KEY_FLOAT if fk else KEY_INTEGER, _bits(empty_key, kb, fk),
                   _bits(empty_value, vb, fv), _bits(erased_key, kb, fk))
        h = C.c_void_p()
        _call("b2co_dmap_create", C.byref(d), C.c_uint64(initial_capacity), _stream(stream), C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.b2co_dmap_destroy(h)
            self._h = None

    def _u64(self, name):
        v = C.c_uint64()
        _call(name, self._h, C.byref(v))
        return v.value

    def Size(self):
        return self._u64("b2co_dmap_size")

    def Capacity(self):
        return self._u64("b2co_dmap_capacity")

    def NumSubmaps(self):
        return self._u64("b2co_dmap_num_submaps")

    def Reserve(self, n, stream=None):
        _call("b2co_dmap_reserve", self._h, C.c_uint64(n), _stream(stream))

    def Insert(self, values, n=None, stream=None, mode=INSERT_EXACT_DEDUP) -> int:
        v = C.c_uint64()
        _call("b2co_dmap_insert", self._h, _ptr(values), C.c_uint64(_OaBase._n(values, n)), C.c_int(mode),
              _stream(stream), C.byref(v))
        return v.value

    def InsertOrAssign(self, values, n=None, stream=None) -> int:
        v = C.c_uint64()
        _call("b2co_dmap_insert_or_assign", self._h, _ptr(values), C.c_uint64(_OaBase._n(values, n)),
              _stream(stream), C.byref(v))
        return v.value

    def Find(self, keys, output_values, n=None, stream=None):
        _call("b2co_dmap_find", self._h, _ptr(keys), _ptr(output_values), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def Contains(self, keys, output_values, n=None, stream=None):
        _call("b2co_dmap_contains", self._h, _ptr(keys), _ptr(output_values), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def Erase(self, keys, n=None, stream=None) -> int:
        v = C.c_uint64()
        _call("b2co_dmap_erase", self._h, _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _stream(stream),
              C.byref(v))
        return v.value

    def Clear(self, stream=None):
        _call("b2co_dmap_clear", self._h, _stream(stream))


class StaticMultiset:
    """StaticMultiset<Key> (include/static_multiset.h), Key int32 or int64;
    device tensors in and out; synchronous like the reference."""

    def __init__(self, capacity, empty_key, key_dtype=None, stream=None):
        import torch
        key_dtype = key_dtype or torch.int64
        self.key_bytes = _dtype_bytes(key_dtype)
        h = C.c_void_p()
        _call("b2co_mset_create", C.c_uint64(capacity), C.c_uint32(self.key_bytes),
              C.c_uint64(_bits(empty_key, self.key_bytes)), _stream(stream), C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.b2co_mset_destroy(h)
            self._h = None

    def _u64(self, name, *args):
        v = C.c_uint64()
        _call(name, self._h, *args, C.byref(v))
        return v.value

    def Capacity(self):
        return self._u64("b2co_mset_capacity")

    def Size(self, stream=None):
        return self._u64("b2co_mset_size")

    def Clear(self, stream=None):
        _call("b2co_mset_clear", self._h, _stream(stream))

    def Insert(self, keys, n=None, stream=None):
        return self._u64("b2co_mset_insert", _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def InsertIf(self, keys, stencil, n=None, stream=None):
        return self._u64("b2co_mset_insert_if", _ptr(keys), _ptr(stencil), C.c_uint64(_OaBase._n(keys, n)),
                         _stream(stream))

    def Contains(self, keys, output, n=None, stream=None):
        _call("b2co_mset_contains", self._h, _ptr(keys), _ptr(output), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def ContainsIf(self, keys, stencil, output, n=None, stream=None):
        _call("b2co_mset_contains_if", self._h, _ptr(keys), _ptr(stencil), _ptr(output),
              C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def Find(self, keys, output, n=None, stream=None):
        _call("b2co_mset_find", self._h, _ptr(keys), _ptr(output), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def FindIf(self, keys, stencil, output, n=None, stream=None):
        _call("b2co_mset_find_if", self._h, _ptr(keys), _ptr(stencil), _ptr(output),
              C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def CountEach(self, keys, output, n=None, stream=None):
        _call("b2co_mset_count_each", self._h, _ptr(keys), _ptr(output), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def CountEachOuter(self, keys, output, n=None, stream=None):
        _call("b2co_mset_count_each_outer", self._h, _ptr(keys), _ptr(output), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def Count(self, keys, n=None, stream=None):
        return self._u64("b2co_mset_count", _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def Retrieve(self, keys, probe_output, match_output, output_capacity, n=None, stream=None):
        return self._u64("b2co_mset_retrieve", _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _ptr(probe_output),
                         _ptr(match_output), C.c_uint64(output_capacity), _stream(stream))

    def RetrieveAll(self, output, output_capacity, stream=None):
        return self._u64("b2co_mset_retrieve_all", _ptr(output), C.c_uint64(output_capacity), _stream(stream))


class StaticMultimap:
    """StaticMultimap<Key, Value> (include/static_multimap.h), int32 / int64;
    inputs are Pair<Key, Value> arrays (pack_pairs); synchronous."""

    def __init__(self, capacity, empty_key, empty_value, key_dtype=None, value_dtype=None, stream=None):
        import torch
        self.key_bytes = _dtype_bytes(key_dtype or torch.int64)
        self.value_bytes = _dtype_bytes(value_dtype or torch.int64)
        h = C.c_void_p()
        _call("b2co_mmap_create", C.c_uint64(capacity), C.c_uint32(self.key_bytes), C.c_uint32(self.value_bytes),
              C.c_uint64(_bits(empty_key, self.key_bytes)), C.c_uint64(_bits(empty_value, self.value_bytes)),
              _stream(stream), C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.b2co_mmap_destroy(h)
            self._h = None

    def _u64(self, name, *args):
        v = C.c_uint64()
        _call(name, self._h, *args, C.byref(v))
        return v.value

    def Capacity(self):
        return self._u64("b2co_mmap_capacity")

    def Size(self, stream=None):
        return self._u64("b2co_mmap_size")

    def Clear(self, stream=None):
        _call("b2co_mmap_clear", self._h, _stream(stream))

    def Insert(self, pairs, n=None, stream=None):
        return self._u64("b2co_mmap_insert", _ptr(pairs), C.c_uint64(_OaBase._n(pairs, n)), _stream(stream))

    def InsertIf(self, pairs, stencil, n=None, stream=None):
        return self._u64("b2co_mmap_insert_if", _ptr(pairs), _ptr(stencil), C.c_uint64(_OaBase._n(pairs, n)),
                         _stream(stream))

    def Contains(self, keys, output, n=None, stream=None):
        _call("b2co_mmap_contains", self._h, _ptr(keys), _ptr(output), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def ContainsIf(self, keys, stencil, output, n=None, stream=None):
        _call("b2co_mmap_contains_if", self._h, _ptr(keys), _ptr(stencil), _ptr(output),
              C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def Find(self, keys, output, n=None, stream=None):
        _call("b2co_mmap_find", self._h, _ptr(keys), _ptr(output), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def FindIf(self, keys, stencil, output, n=None, stream=None):
        _call("b2co_mmap_find_if", self._h, _ptr(keys), _ptr(stencil), _ptr(output),
              C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def Count(self, keys, n=None, stream=None):
        return self._u64("b2co_mmap_count", _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def Retrieve(self, keys, key_output, value_output, output_capacity, n=None, stream=None):
        return self._u64("b2co_mmap_retrieve", _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _ptr(key_output),
                         _ptr(value_output), C.c_uint64(output_capacity), _stream(stream))

    def RetrieveAll(self, key_output, value_output, output_capacity, stream=None):
        return self._u64("b2co_mmap_retrieve_all", _ptr(key_output), _ptr(value_output),
                         C.c_uint64(output_capacity), _stream(stream))


def roaring_parse(data: bytes, key_bytes: int = 4, bounded: bool = True):
    """(num_keys, size_bytes) of a serialized portable Roaring bitmap (host
    only; the validation RoaringBitmap's constructor runs)."""
    nk, sb = C.c_uint64(), C.c_uint64()
    buf = C.create_string_buffer(bytes(data), len(data))
    _call("b2co_roaring_parse", buf, C.c_uint64(len(data) if bounded else 2**64 - 1), C.c_uint32(key_bytes),
          C.byref(nk), C.byref(sb))
    return nk.value, sb.value


class RoaringBitmap:
    """RoaringBitmap<Key> (include/roaring_bitmap.h) over a portable
    serialized bitmap held in host memory; Key uint32 (key_bytes 4) or uint64
    (key_bytes 8, the 64-bit bucketed form)."""

    def __init__(self, data: bytes, key_bytes: int = 4, bounded: bool = True, stream=None):
        self.key_bytes = key_bytes
        h = C.c_void_p()
        buf = C.create_string_buffer(bytes(data), len(data))
        _call("b2co_roaring_create", buf, C.c_uint64(len(data) if bounded else 2**64 - 1), C.c_uint32(key_bytes),
              _stream(stream), C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.b2co_roaring_destroy(h)
            self._h = None

    def Contains(self, keys, output, n=None, stream=None):
        _call("b2co_roaring_contains", self._h, _ptr(keys), _ptr(output), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def ContainsAsync(self, keys, output, n=None, stream=None):
        _call("b2co_roaring_contains_async", self._h, _ptr(keys), _ptr(output), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def Size(self) -> int:
        v = C.c_uint64()
        _call("b2co_roaring_size", self._h, C.byref(v))
        return v.value

    def Empty(self) -> bool:
        return self.Size() == 0

    def SizeBytes(self) -> int:
        v = C.c_uint64()
        _call("b2co_roaring_size_bytes", self._h, C.byref(v))
        return v.value

    def Data(self) -> int:
        p = C.c_void_p()
        _call("b2co_roaring_data", self._h, C.byref(p))
        return p.value

    def bytes(self) -> bytes:
        """The device copy of the serialized bitmap, read back."""
        return _device_bytes(self.Data(), self.SizeBytes()).tobytes()


class BloomFilter:
    """BloomFilter<Key, Extent, BloomFilterPolicy<Key, xxhash_64<Key>, uint32_t,
    WordsPerBlock, PatternBits>> (include/bloom_filter.h:37-39,
    bloom_filter_policy.h:42-181); the defaults (8, 8) are the reference's
    default policy and ArrowFilterPolicy."""

    def __init__(self, num_blocks, key_dtype=None, seed=0, stream=None, words_per_block=8, pattern_bits=8):
        import torch
        key_dtype = key_dtype or torch.uint64
        self.key_bytes = _dtype_bytes(key_dtype)
        h = C.c_void_p()
        _call("b2co_bloom_create_policy", C.c_uint64(num_blocks), C.c_uint32(self.key_bytes), C.c_uint64(seed),
              C.c_uint32(words_per_block), C.c_uint32(pattern_bits), _stream(stream), C.byref(h))
        self._h = h
        self.num_blocks = num_blocks
        self.words_per_block = words_per_block
        self.pattern_bits = pattern_bits

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.b2co_bloom_destroy(h)
            self._h = None

    def Data(self) -> int:
        p = C.c_void_p()
        _call("b2co_bloom_data", self._h, C.byref(p))
        return p.value

    def set_add_mode(self, mode: int):
        """How the default policy's Add updates the filter (the bits are the same either way):
        BLOOM_ADD_ATOMIC (64-bit atomics per key), BLOOM_ADD_BULK (one 32-byte TMA bulk OR per key),
        BLOOM_ADD_PARTITIONED (keys routed by filter slice, each slice built in shared memory) or
        BLOOM_ADD_AUTO (the default: partitioned for filters of at least 64 MiB and batches of at least 8 keys
        per block, else bulk)."""
        _call("b2co_bloom_set_add_mode", self._h, C.c_int(mode))

    def words(self) -> np.ndarray:
        """The filter's words copied to the host (uint32, words_per_block per block)."""
        return _device_bytes(self.Data(), self.num_blocks * self.words_per_block * 4).view(np.uint32)

    def Clear(self, stream=None):
        _call("b2co_bloom_clear", self._h, _stream(stream))

    def ClearAsync(self, stream=None):
        _call("b2co_bloom_clear_async", self._h, _stream(stream))

    def Add(self, keys, n=None, stream=None):
        _call("b2co_bloom_add", self._h, _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def AddAsync(self, keys, n=None, stream=None):
        _call("b2co_bloom_add_async", self._h, _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def AddIf(self, keys, stencil, n=None, stream=None):
        _call("b2co_bloom_add_if", self._h, _ptr(keys), _ptr(stencil), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def Contains(self, keys, output_values, n=None, stream=None):
        _call("b2co_bloom_contains", self._h, _ptr(keys), _ptr(output_values), C.c_uint64(_OaBase._n(keys, n)),
              _stream(stream))

    def ContainsAsync(self, keys, output_values, n=None, stream=None):
        _call("b2co_bloom_contains_async", self._h, _ptr(keys), _ptr(output_values),
              C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def ContainsIf(self, keys, stencil, output_values, n=None, stream=None):
        _call("b2co_bloom_contains_if", self._h, _ptr(keys), _ptr(stencil), _ptr(output_values),
              C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def Merge(self, other, stream=None):
        _call("b2co_bloom_merge", self._h, other._h, _stream(stream))

    def MergeAsync(self, other, stream=None):
        _call("b2co_bloom_merge_async", self._h, other._h, _stream(stream))

    def Intersect(self, other, stream=None):
        _call("b2co_bloom_intersect", self._h, other._h, _stream(stream))


class HyperLogLog:
    """HyperLogLog<Key> for int32/int64 keys (include/hyperloglog.h:23-59)."""

    def __init__(self, precision, key_dtype=None, stream=None):
        import torch
        key_dtype = key_dtype or torch.int64
        self.key_bytes = _dtype_bytes(key_dtype)
        h = C.c_void_p()
        _call("b2co_hll_create", C.c_uint32(precision), C.c_uint32(self.key_bytes), _stream(stream), C.byref(h))
        self._h = h
        self.precision = precision

    @classmethod
    def CreateWithSketchSizeKB(cls, kb, key_dtype=None, stream=None):
        p = C.c_uint32()
        _call("b2co_hll_precision_for_sketch_kb", C.c_uint32(kb), C.byref(p))
        return cls(p.value, key_dtype, stream)

    @classmethod
    def CreateWithPrecision(cls, precision, key_dtype=None, stream=None):
        return cls(precision, key_dtype, stream)

    @classmethod
    def CreateWithStandardDeviation(cls, deviation, key_dtype=None, stream=None):
        p = C.c_uint32()
        _call("b2co_hll_precision_for_deviation", C.c_double(deviation), C.byref(p))
        return cls(p.value, key_dtype, stream)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.b2co_hll_destroy(h)
            self._h = None

    def SketchSizeKB(self):
        return (1 << self.precision) // 1024

    def Data(self) -> int:
        p = C.c_void_p()
        _call("b2co_hll_data", self._h, C.byref(p))
        return p.value

    def registers(self) -> np.ndarray:
        """The 2^precision register bytes copied to the host."""
        return _device_bytes(self.Data(), 1 << self.precision)

    def Clear(self, stream=None):
        _call("b2co_hll_clear", self._h, _stream(stream))

    def Add(self, keys, n=None, stream=None):
        _call("b2co_hll_add", self._h, _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def AddAsync(self, keys, n=None, stream=None):
        _call("b2co_hll_add_async", self._h, _ptr(keys), C.c_uint64(_OaBase._n(keys, n)), _stream(stream))

    def Merge(self, other, stream=None):
        _call("b2co_hll_merge", self._h, other._h, _stream(stream))

    def Estimate(self, stream=None) -> int:
        v = C.c_uint64()
        _call("b2co_hll_estimate", self._h, _stream(stream), C.byref(v))
        return v.value

    def Histogram(self, stream=None) -> np.ndarray:
        h = np.zeros(65, dtype=np.uint32)
        _call("b2co_hll_histogram", self._h, _stream(stream), C.c_void_p(h.ctypes.data))
        return h


def tune_cache_save(path: str):
    _call("b2co_tune_cache_save", path.encode())


def tune_cache_load(path: str):
    _call("b2co_tune_cache_load", path.encode())


def tune_cache_clear():
    _call("b2co_tune_cache_clear")


def hll_finalize(precision: int, hist) -> int:
    hist = np.ascontiguousarray(hist, dtype=np.uint32)
    v = C.c_uint64()
    _call("b2co_hll_finalize", C.c_uint32(precision), C.c_void_p(hist.ctypes.data), C.byref(v))
    return v.value


def hll_bias_data(precision: int):
    raw, bias = C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
    n, thr = C.c_uint32(), C.c_double()
    _call("b2co_hll_bias_data", C.c_uint32(precision), C.byref(raw), C.byref(bias), C.byref(n), C.byref(thr))
    return (np.ctypeslib.as_array(raw, shape=(n.value,)).copy(), np.ctypeslib.as_array(bias, shape=(n.value,)).copy(),
            thr.value)
