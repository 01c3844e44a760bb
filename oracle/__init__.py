"""CPU oracle for the ops-collections bulk-container hot path (ctypes + numpy).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path and the timed
CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg import this package; the product (``ops-collections_b200``)
never does.

The algorithms live in ``oracle.c`` (a sequential C restatement of the
reference, each function citing the reference file:line it follows); this
module only marshals numpy arrays.  The oracle is pinned by
``tests/golden/*.json`` -- known answers from the reference's own tests and
outputs of the reference's host headers recorded by ``tests/golden/make_golden.py``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "liboracle.so")

HASH_XXH32, HASH_MURMUR3_32, HASH_FMIX, HASH_XXH64 = 0, 1, 2, 3
PROBE_LINEAR, PROBE_DOUBLE = 0, 1
FAILED, SUCCESS, DUPLICATE = 0, 1, 2


def build() -> str:
    """Compile liboracle.so with gcc (oracle/Makefile) if it is missing or stale."""
    src = os.path.join(_HERE, "oracle.c")
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        u32, u64, i32, vp, sz = C.c_uint32, C.c_uint64, C.c_int, C.c_void_p, C.c_size_t
        sig = {
            "orc_xxh32": (u32, [vp, sz, u32]),
            "orc_xxh64": (u64, [vp, sz, u64]),
            "orc_murmur3_32": (u32, [vp, sz, u32]),
            "orc_fmix32": (u32, [u32, u32]),
            "orc_fmix64": (u64, [u64, u64]),
            "orc_probe_hash": (u32, [i32, u64, u32, u32]),
            "orc_prime_table_size": (u64, []),
            "orc_prime_table_entry": (u64, [u64]),
            "orc_prime_at_least": (u64, [u64]),
            "orc_valid_capacity": (u64, [u64, u32, i32]),
            "orc_slot_layout": (None, [u32, u32, vp, vp]),
            "orc_table_clear": (None, [vp]),
            "orc_insert": (u64, [vp, vp, vp, vp, u64]),
            "orc_insert_or_assign": (u64, [vp, vp, vp, u64, vp]),
            "orc_assign_if": (None, [vp, vp, vp, vp, u64]),
            "orc_insert_and_find": (None, [vp, vp, vp, u64, vp, vp]),
            "orc_find": (None, [vp, vp, vp, u64, vp, vp]),
            "orc_contains": (None, [vp, vp, vp, u64, vp, vp]),
            "orc_find_parallel": (None, [vp, vp, u64, vp, i32]),
            "orc_contains_parallel": (None, [vp, vp, u64, vp, i32]),
            "orc_key_equal": (i32, [i32, u32, u64, u64]),
            "orc_pairs_match": (None, [vp, vp, vp, vp, vp, i32]),
            "orc_group_check": (u64, [u64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32]),
            "orc_erase": (u64, [vp, vp, u64]),
            "orc_count": (u64, [vp, vp, u64]),
            "orc_bloom_add": (None, [vp, u64, vp, u32, u64, u64]),
            "orc_bloom_contains": (None, [vp, u64, vp, u32, u64, u64, vp]),
            "orc_bloom_contains_parallel": (None, [vp, u64, vp, u32, u64, u64, vp, i32]),
            "orc_bloom_policy_valid": (i32, [u32, u32]),
            "orc_bloom_word_pattern": (u32, [u32, u32, u32]),
            "orc_bloom_add_policy": (None, [vp, u64, u32, u32, vp, u32, u64, u64]),
            "orc_bloom_contains_policy": (None, [vp, u64, u32, u32, vp, u32, u64, u64, vp, i32]),
            "orc_hll_add": (None, [vp, u32, vp, u32, u64]),
            "orc_hll_add_parallel": (None, [vp, u32, vp, u32, u64, i32]),
            "orc_hll_merge": (None, [vp, vp, u32]),
            "orc_hll_histogram": (None, [vp, u32, vp]),
            "orc_hll_finalize": (u64, [u32, vp, vp, vp, i32, C.c_double]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


_UINT = {2: np.uint16, 4: np.uint32, 8: np.uint64}
_FLOAT = {2: np.float16, 4: np.float32, 8: np.float64}


def _bits(x, nbytes: int) -> int:
    """Bit pattern of a sentinel as an unsigned value: two's complement for
    integers, the IEEE encoding of that width for floats."""
    if isinstance(x, (float, np.floating)):
        return int(np.array([x], dtype=_FLOAT[nbytes]).view(_UINT[nbytes])[0])
    return int(x) & ((1 << (8 * nbytes)) - 1)


KEY_INT, KEY_FLOAT = 0, 1


# ---- hashes ---------------------------------------------------------------

def xxh32(key_bytes: bytes, seed: int = 0) -> int:
    return lib().orc_xxh32(key_bytes, len(key_bytes), seed)


def xxh64(key_bytes: bytes, seed: int = 0) -> int:
    return lib().orc_xxh64(key_bytes, len(key_bytes), seed)


def murmur3_32(key_bytes: bytes, seed: int = 0) -> int:
    return lib().orc_murmur3_32(key_bytes, len(key_bytes), seed)


def fmix32(k: int, seed: int = 0) -> int:
    return lib().orc_fmix32(k, seed)


def fmix64(k: int, seed: int = 0) -> int:
    return lib().orc_fmix64(k, seed)


def probe_hash(kind: int, key_bits: int, key_bytes: int, seed: int) -> int:
    return lib().orc_probe_hash(kind, key_bits, key_bytes, seed)


def key_equal(key_kind: int, key_bytes: int, a_bits: int, b_bits: int) -> bool:
    """KeyEqual of a table of that key kind (KEY_INT bitwise, KEY_FLOAT IEEE ==) on bit patterns."""
    return bool(lib().orc_key_equal(key_kind, key_bytes, a_bits, b_bits))


def prime_table():
    n = lib().orc_prime_table_size()
    return np.array([lib().orc_prime_table_entry(i) for i in range(n)], dtype=np.uint64)


def prime_at_least(n: int) -> int:
    return lib().orc_prime_at_least(n)


def valid_capacity(request: int, bucket_size: int, probing: int) -> int:
    return lib().orc_valid_capacity(request, bucket_size, probing)


# ---- open-addressing table --------------------------------------------------

class _CTable(C.Structure):
    _fields_ = [
        ("slots", C.c_void_p), ("capacity", C.c_uint32), ("key_bytes", C.c_uint32),
        ("value_bytes", C.c_uint32), ("slot_bytes", C.c_uint32), ("value_offset", C.c_uint32),
        ("bucket_size", C.c_uint32), ("probing", C.c_int), ("hash_kind", C.c_int),
        ("empty_key", C.c_uint64), ("empty_value", C.c_uint64), ("erased_key", C.c_uint64),
        ("key_kind", C.c_int),
    ]


def slot_layout(key_bytes: int, value_bytes: int):
    sb, vo = C.c_uint32(), C.c_uint32()
    lib().orc_slot_layout(key_bytes, value_bytes, C.byref(sb), C.byref(vo))
    return sb.value, vo.value


class Table:
    """A host open-addressing table with the reference's layout and semantics.

    ``key_dtype``/``value_dtype`` are numpy integer or floating dtypes of 2, 4
    or 8 bytes; ``value_dtype`` None makes a set.  Floating-point keys match
    with IEEE ``==`` (so -0.0 finds +0.0 and NaN finds nothing); sentinels are
    always compared bitwise.  ``capacity`` is the already-valid slot count (use
    :func:`valid_capacity` on a request first).
    """

    def __init__(self, key_dtype, value_dtype, capacity: int, bucket_size: int = 5,
                 probing: int = PROBE_DOUBLE, hash_kind: int = HASH_XXH32,
                 empty_key=-1, empty_value=-1, erased_key=None):
        self.kdt = np.dtype(key_dtype)
        self.vdt = None if value_dtype is None else np.dtype(value_dtype)
        kb = self.kdt.itemsize
        vb = 0 if self.vdt is None else self.vdt.itemsize
        sb, vo = slot_layout(kb, vb)
        self.slots = np.zeros(capacity * sb, dtype=np.uint8)
        fk = self.kdt.kind == "f"
        if fk and not isinstance(empty_key, (float, np.floating)):
            empty_key = float(empty_key)
        if fk and erased_key is not None and not isinstance(erased_key, (float, np.floating)):
            erased_key = float(erased_key)
        if self.vdt is not None and self.vdt.kind == "f" and not isinstance(empty_value, (float, np.floating)):
            empty_value = float(empty_value)
        ek = _bits(empty_key, kb)
        self.c = _CTable(
            _p(self.slots), capacity, kb, vb, sb, vo, bucket_size, probing, hash_kind,
            ek, _bits(empty_value, vb) if vb else 0,
            ek if erased_key is None else _bits(erased_key, kb), KEY_FLOAT if fk else KEY_INT)
        lib().orc_table_clear(C.byref(self.c))

    @property
    def capacity(self) -> int:
        return self.c.capacity

    def _out_dtype(self):
        return self.vdt if self.vdt is not None else self.kdt

    def _k(self, keys):
        return np.ascontiguousarray(keys, dtype=self.kdt)

    def _v(self, values, n):
        if self.vdt is None:
            return None
        return np.ascontiguousarray(values, dtype=self.vdt)

    def _s(self, stencil):
        return None if stencil is None else np.ascontiguousarray(stencil, dtype=np.uint8)

    def insert(self, keys, values=None, stencil=None) -> int:
        k = self._k(keys)
        v = self._v(values, len(k))
        s = self._s(stencil)
        return lib().orc_insert(C.byref(self.c), _p(k), _p(v), _p(s), len(k))

    def insert_or_assign(self, keys, values):
        k, v = self._k(keys), self._v(values, len(keys))
        asg = C.c_uint64()
        f = lib().orc_insert_or_assign(C.byref(self.c), _p(k), _p(v), len(k), C.byref(asg))
        return f, asg.value

    def assign_if(self, keys, values, stencil=None):
        k, v, s = self._k(keys), self._v(values, len(keys)), self._s(stencil)
        lib().orc_assign_if(C.byref(self.c), _p(k), _p(v), _p(s), len(k))

    def insert_and_find(self, keys, values=None):
        k = self._k(keys)
        v = self._v(values, len(k))
        found = np.empty(len(k), dtype=self._out_dtype())
        ins = np.empty(len(k), dtype=np.uint8)
        lib().orc_insert_and_find(C.byref(self.c), _p(k), _p(v), len(k), _p(found), _p(ins))
        return found, ins

    def find(self, keys, stencil=None):
        k, s = self._k(keys), self._s(stencil)
        out = np.empty(len(k), dtype=self._out_dtype())
        win = np.empty(len(k), dtype=np.uint32)
        lib().orc_find(C.byref(self.c), _p(k), _p(s), len(k), _p(out), _p(win))
        return out, win

    def find_parallel(self, keys, threads: int = 0):
        k = self._k(keys)
        out = np.empty(len(k), dtype=self._out_dtype())
        lib().orc_find_parallel(C.byref(self.c), _p(k), len(k), _p(out), threads)
        return out

    def contains_parallel(self, keys, threads: int = 0):
        k = self._k(keys)
        out = np.empty(len(k), dtype=np.uint8)
        lib().orc_contains_parallel(C.byref(self.c), _p(k), len(k), _p(out), threads)
        return out

    def same_pairs(self, other: "Table", threads: int = 0):
        """(equal, occupied_self, occupied_other, mismatches): whether ``other``
        (e.g. a device table's dump) stores exactly this table's pair set.
        ``self``'s keys must be distinct (true of any table built by the oracle)."""
        oa, ob, mm = C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().orc_pairs_match(C.byref(self.c), C.byref(other.c), C.byref(oa), C.byref(ob), C.byref(mm), threads)
        return mm.value == 0 and oa.value == ob.value, oa.value, ob.value, mm.value

    def contains(self, keys, stencil=None):
        k, s = self._k(keys), self._s(stencil)
        out = np.empty(len(k), dtype=np.uint8)
        win = np.empty(len(k), dtype=np.uint32)
        lib().orc_contains(C.byref(self.c), _p(k), _p(s), len(k), _p(out), _p(win))
        return out, win

    def erase(self, keys) -> int:
        k = self._k(keys)
        return lib().orc_erase(C.byref(self.c), _p(k), len(k))

    def count(self, keys) -> int:
        k = self._k(keys)
        return lib().orc_count(C.byref(self.c), _p(k), len(k))

    def load_slots(self, raw: np.ndarray):
        """Replace the slot bytes with a dump of a device table of the same layout."""
        raw = np.ascontiguousarray(raw).view(np.uint8).reshape(-1)
        assert raw.size == self.slots.size
        self.slots[:] = raw

    def slot_keys_values(self):
        """(keys, values) arrays of every slot, as stored."""
        sb, vo = self.c.slot_bytes, self.c.value_offset
        s = self.slots.reshape(-1, sb)
        keys = s[:, :self.kdt.itemsize].copy().view(self.kdt).reshape(-1)
        if self.vdt is None:
            return keys, None
        vals = s[:, vo:vo + self.vdt.itemsize].copy().view(self.vdt).reshape(-1)
        return keys, vals

    def pairs(self):
        """The stored pair set: sorted (key bits, value bits) rows of occupied
        slots (unsigned bit patterns, so floating-point keys sort and compare
        exactly)."""
        keys, vals = self.slot_keys_values()
        ut = _UINT[self.kdt.itemsize]
        kb = keys.view(ut)
        occ = kb != ut(self.c.empty_key)
        if self.c.erased_key != self.c.empty_key:
            occ &= kb != ut(self.c.erased_key)
        if vals is None:
            return np.sort(kb[occ]).astype(np.uint64)
        k, v = kb[occ].astype(np.uint64), vals[occ].view(_UINT[self.vdt.itemsize]).astype(np.uint64)
        order = np.lexsort((v, k))
        return np.stack([k[order], v[order]], axis=1)


def group_check(caps, shape: Table, slab: np.ndarray, keys, values, ins_off, queries, q_off, threads: int = 0):
    """The batched pattern checked table by table: every table is rebuilt by
    the oracle from its own inserts (tables in parallel), its stored set is
    compared with its segment of ``slab`` (the device group's slot dump, tables
    back to back), and its queries are answered.  Returns (bad_tables,
    first_bad_table_or_None, expected_find_outputs)."""
    caps = np.ascontiguousarray(caps, dtype=np.uint64)
    slot_off = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.uint64)
    k = np.ascontiguousarray(keys, dtype=shape.kdt)
    v = None if shape.vdt is None else np.ascontiguousarray(values, dtype=shape.vdt)
    q = np.ascontiguousarray(queries, dtype=shape.kdt)
    io = np.ascontiguousarray(ins_off, dtype=np.uint64)
    qo = np.ascontiguousarray(q_off, dtype=np.uint64)
    raw = np.ascontiguousarray(slab).view(np.uint8).reshape(-1)
    assert raw.size == int(caps.sum()) * shape.c.slot_bytes
    out = np.empty(len(q), dtype=shape._out_dtype())
    first = C.c_uint64()
    bad = lib().orc_group_check(len(caps), _p(caps), _p(slot_off), _p(raw), C.byref(shape.c), _p(k), _p(v), _p(io),
                                _p(q), _p(qo), _p(out), C.byref(first), threads)
    return int(bad), (None if bad == 0 else int(first.value)), out


# ---- Bloom filter -----------------------------------------------------------

def bloom_policy_valid(words_per_block: int, pattern_bits: int) -> bool:
    return bool(lib().orc_bloom_policy_valid(words_per_block, pattern_bits))


def bloom_word_patterns(words_per_block: int, pattern_bits: int, lower_hash: int):
    """The per-word bit patterns one key sets (its 32-bit lower hash)."""
    bpw = pattern_bits // words_per_block
    return [lib().orc_bloom_word_pattern(w, bpw, lower_hash) for w in range(words_per_block)]


def bloom_add(words: np.ndarray, num_blocks: int, keys: np.ndarray, seed: int = 0, words_per_block: int = 8,
              pattern_bits: int = 8):
    """Adds keys to a host word array of num_blocks * words_per_block uint32."""
    keys = np.ascontiguousarray(keys)
    lib().orc_bloom_add_policy(_p(words), num_blocks, words_per_block, pattern_bits, _p(keys), keys.dtype.itemsize,
                               len(keys), seed)


def bloom_contains(words: np.ndarray, num_blocks: int, keys: np.ndarray, seed: int = 0, threads: int = 1,
                   words_per_block: int = 8, pattern_bits: int = 8):
    keys = np.ascontiguousarray(keys)
    out = np.empty(len(keys), dtype=np.uint8)
    lib().orc_bloom_contains_policy(_p(words), num_blocks, words_per_block, pattern_bits, _p(keys),
                                    keys.dtype.itemsize, len(keys), seed, _p(out), threads)
    return out


# ---- HyperLogLog --------------------------------------------------------------

def hll_add(registers: np.ndarray, precision: int, keys: np.ndarray, threads: int = 1):
    keys = np.ascontiguousarray(keys)
    if threads == 1:
        lib().orc_hll_add(_p(registers), precision, _p(keys), keys.dtype.itemsize, len(keys))
    else:
        lib().orc_hll_add_parallel(_p(registers), precision, _p(keys), keys.dtype.itemsize, len(keys), threads)


def hll_merge(dst: np.ndarray, src: np.ndarray, precision: int):
    lib().orc_hll_merge(_p(dst), _p(src), precision)


def hll_histogram(registers: np.ndarray, precision: int) -> np.ndarray:
    h = np.zeros(65, dtype=np.uint32)
    lib().orc_hll_histogram(_p(registers), precision, _p(h))
    return h


def hll_finalize(precision: int, hist: np.ndarray, raw: np.ndarray, bias: np.ndarray, threshold: float) -> int:
    hist = np.ascontiguousarray(hist, dtype=np.uint32)
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    bias = np.ascontiguousarray(bias, dtype=np.float64)
    return lib().orc_hll_finalize(precision, _p(hist), _p(raw), _p(bias), len(raw), threshold)
