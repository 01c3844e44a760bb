"""CPU-only checks of the C-ABI library: it loads, exports every symbol that
include/b2co.h declares, and its host-side logic (capacity rule, argument
validation, HLL++ finalizer and its data) matches the reference.  No kernel
is launched."""
import ctypes as C
import hashlib
import json
import os
import re

import numpy as np
import pytest

import b2co
import oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(REPO, "tests", "golden")


def header_symbols():
    names = set()
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(REPO, "include", fn)).read()
            names |= set(re.findall(r"^[A-Za-z_][\w\s\*]*?\b(b2co_\w+)\s*\(", src, re.M))
    return names


def test_library_exports_every_declared_symbol():
    names = header_symbols()
    assert len(names) > 60
    L = b2co.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_status_strings():
    L = b2co.lib()
    assert b"sm_100a" in L.b2co_version()
    assert L.b2co_status_string(b2co.ERANGE) == b"length error"


def load(name):
    with open(os.path.join(GOLD, name + ".json")) as f:
        return json.load(f)


def test_capacity_rule_matches_reference():
    g = load("capacity")
    for row in g["tables"]:
        probing = b2co.PROBE_DOUBLE if row["double_hashing"] else b2co.PROBE_LINEAR
        got = [b2co.valid_capacity(r, row["bucket_size"], probing) for r in g["requests"]]
        assert got == row["capacities"], (row["bucket_size"], row["double_hashing"])
    # beyond the last table prime: MakeValidExtent throws invalid_argument
    with pytest.raises(b2co.InvalidArgument):
        b2co.valid_capacity(int(g["prime_last"][-1]) * 5 + 6, 5, b2co.PROBE_DOUBLE)


def test_create_validation_errors_before_any_device_work():
    L = b2co.lib()
    h = C.c_void_p()
    for kb, vb, b, pr, hs, res in [(3, 4, 5, 1, 0, 0), (4, 2, 5, 1, 0, 0), (4, 4, 3, 1, 0, 0), (4, 4, 5, 7, 0, 0),
                                   (4, 4, 5, 1, 9, 0), (4, 4, 5, 1, 0, 2)]:
        d = b2co.OaDesc(kb, vb, b, pr, hs, res, 0xffffffff, 0xffffffff, 0xffffffff)
        assert L.b2co_oa_create(C.byref(d), C.c_uint64(100), None, C.byref(h)) == b2co.EINVAL
        assert L.b2co_last_error()
    # a capacity beyond the kernels' 32-bit slot index is a length error
    d = b2co.OaDesc(8, 8, 1, 0, 0, 0, 0, 0, 0)
    assert L.b2co_oa_create(C.byref(d), C.c_uint64(1 << 33), None, C.byref(h)) == b2co.ERANGE
    # BloomFilter: zero blocks / more than 2^32-1 blocks (bloom_filter_lifecycle.inl:24-29)
    assert L.b2co_bloom_create(C.c_uint64(0), 8, C.c_uint64(0), None, C.byref(h)) == b2co.EINVAL
    assert L.b2co_bloom_create(C.c_uint64(1 << 32), 8, C.c_uint64(0), None, C.byref(h)) == b2co.ERANGE
    # HyperLogLog precision range (hyperloglog.inl:125-130)
    assert L.b2co_hll_create(12, 8, None, C.byref(h)) == b2co.EINVAL
    assert L.b2co_hll_create(19, 8, None, C.byref(h)) == b2co.EINVAL
    # DynamicMap: emptyKey == erasedKey (dynamic_map.h:107-109)
    d = b2co.OaDesc(4, 4, 5, 0, 1, 0, 0xffffffff, 0xffffffff, 0xffffffff)
    assert L.b2co_dmap_create(C.byref(d), C.c_uint64(100), None, C.byref(h)) == b2co.EINVAL


def test_hll_precision_helpers():
    p = C.c_uint32()
    L = b2co.lib()
    for kb, want in [(8, 13), (16, 14), (64, 16), (256, 18)]:
        assert L.b2co_hll_precision_for_sketch_kb(kb, C.byref(p)) == 0 and p.value == want
    for bad in (4, 12, 512):
        assert L.b2co_hll_precision_for_sketch_kb(bad, C.byref(p)) == b2co.EINVAL
    for dev, want in [(0.05, 13), (1.04 / 128, 14), (0.0041, 16)]:
        assert L.b2co_hll_precision_for_deviation(C.c_double(dev), C.byref(p)) == 0 and p.value == want
    assert L.b2co_hll_precision_for_deviation(C.c_double(0.001), C.byref(p)) == b2co.EINVAL


def test_hll_bias_data_pinned_to_reference():
    g = load("hll")
    for p in range(13, 19):
        raw, bias, thr = b2co.hll_bias_data(p)
        t = g["tables"][str(p)]
        assert len(raw) == t["points"] and thr == t["threshold"]
        assert hashlib.sha256(raw.tobytes() + bias.tobytes()).hexdigest() == t["sha256_raw_then_bias_f64le"]


def test_hll_finalizer_matches_reference_and_oracle():
    g = load("hll")
    for c in g["finalizer_cases"]:
        p = c["precision"]
        hist = np.array(c["hist"], dtype=np.uint32)
        assert b2co.hll_finalize(p, hist) == c["estimate"]
        raw, bias, thr = b2co.hll_bias_data(p)
        assert oracle.hll_finalize(p, hist, raw, bias, thr) == c["estimate"]


def test_fastmod_is_exact():
    """The kernels' remainder a mod d = mulhi64((2^64-1)//d + 1) * a mod 2^64, d) for 32-bit a, d."""
    rng = np.random.default_rng(5)
    ds = [1, 2, 3, 4, 5, 7, 31, 32, 33, 524347, 53745631, 2**31 - 1, 2**31, 2**32 - 5, 2**32 - 1]
    ds += [int(x) for x in rng.integers(1, 2**32, size=200, dtype=np.uint64)]
    a_s = [0, 1, 2, 2**31, 2**32 - 1] + [int(x) for x in rng.integers(0, 2**32, size=200, dtype=np.uint64)]
    for d in ds:
        m = ((2**64 - 1) // d + 1) % 2**64
        for a in a_s:
            assert ((m * a % 2**64) * d) >> 64 == a % d, (a, d)


def test_device_key_primitives_on_host_match_reference():
    """The kernels' hash and key comparison (include/b2co/device.cuh), evaluated
    on the host through the library, against the reference's own outputs."""
    import json
    L = b2co.lib()
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    g = json.load(open(os.path.join(here, "hashes.json")))
    out = C.c_uint32()
    for r in g["vectors16"]:
        for hk, name in ((b2co.HASH_XXH32, "xxh32"), (b2co.HASH_MURMUR3_32, "murmur3_32"), (b2co.HASH_XXH64, "xxh64")):
            assert L.b2co_probe_hash(hk, 2, C.c_uint64(r["key"]), r["seed"], C.byref(out)) == 0
            assert out.value == r[name] & 0xFFFFFFFF, (name, r)
    for r in g["vectors"][:200]:
        for hk, name in ((b2co.HASH_XXH32, "xxh32"), (b2co.HASH_MURMUR3_32, "murmur3_32"), (b2co.HASH_XXH64, "xxh64"),
                         (b2co.HASH_FMIX, "fmix")):
            assert L.b2co_probe_hash(hk, r["key_bytes"], C.c_uint64(r["key"]), r["seed"], C.byref(out)) == 0
            assert out.value == r[name] & 0xFFFFFFFF, (name, r)
    assert L.b2co_probe_hash(b2co.HASH_FMIX, 2, C.c_uint64(1), 0, C.byref(out)) == b2co.EINVAL
    eq = C.c_int()
    for r in json.load(open(os.path.join(here, "keys.json")))["float_key_comparisons"]:
        assert L.b2co_key_equal(1, r["key_bytes"], C.c_uint64(r["a"]), C.c_uint64(r["b"]), C.byref(eq)) == 0
        assert eq.value == r["equal"], r
        assert L.b2co_key_equal(0, r["key_bytes"], C.c_uint64(r["a"]), C.c_uint64(r["b"]), C.byref(eq)) == 0
        assert eq.value == int(r["a"] == r["b"]), r


def test_two_byte_and_float_layouts_validate():
    """Descriptor checks of the new layouts, without touching the GPU."""
    L = b2co.lib()
    h = C.c_void_p()
    for kb, vb, kind, hk in [(2, 4, 0, 0), (4, 2, 0, 0), (8, 2, 0, 0), (2, 8, 1, 0), (2, 0, 0, b2co.HASH_FMIX),
                             (4, 4, 2, 0), (3, 0, 0, 0)]:
        d = b2co.OaDesc(kb, vb, 5, 1, hk, kind, 0xFFFF, 0xFFFF, 0xFFFF)
        assert L.b2co_oa_create(C.byref(d), C.c_uint64(100), None, C.byref(h)) == b2co.EINVAL, (kb, vb, kind, hk)
    assert b2co.slot_bytes(2, 2) == 4 and b2co.slot_bytes(2, 0) == 2 and b2co.slot_bytes(4, 4) == 8
    assert b2co.slot_bytes(4, 8) == 16 and b2co.slot_bytes(8, 4) == 16 and b2co.slot_bytes(8, 8) == 16
    for kb, vb in [(2, 0), (2, 2), (4, 0), (4, 4), (4, 8), (8, 4), (8, 8)]:
        assert oracle.slot_layout(kb, vb)[0] == b2co.slot_bytes(kb, vb)


def test_tune_cache_file_round_trip(tmp_path):
    """The batched pattern's autotune cache persists as a text file: entries
    load, unknown lines and comments are skipped, and a save writes them back."""
    src = tmp_path / "in.txt"
    src.write_text("# op key_bytes payload_bytes bucket log2_capacity lanes keys_per_tile block ms\n"
                   "group_find 4 4 5 15 4 2 256 1.2500\nsomething_else 1 2 3\n"
                   "group_find 8 8 5 20 8 4 128 3.0000\n")
    b2co.tune_cache_clear()
    b2co.tune_cache_load(str(src))
    dst = tmp_path / "out.txt"
    b2co.tune_cache_save(str(dst))
    rows = [ln for ln in dst.read_text().splitlines() if not ln.startswith("#")]
    assert rows == ["group_find 4 4 5 15 4 2 256 1.2500", "group_find 8 8 5 20 8 4 128 3.0000"]
    b2co.tune_cache_clear()
    b2co.tune_cache_save(str(dst))
    assert [ln for ln in dst.read_text().splitlines() if not ln.startswith("#")] == []
    with pytest.raises(b2co.InvalidArgument):
        b2co.tune_cache_load(str(tmp_path / "missing.txt"))
