"""Pins the CPU oracle against the reference: known answers from the reference's
own tests and outputs of the reference's host headers (tests/golden/*.json,
made by tests/golden/make_golden.py).  CPU only."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLD, name + ".json")) as f:
        return json.load(f)


def kbytes(k, n):
    return int(k).to_bytes(n, "little")


def test_reference_hash_known_answers():
    kat = load("hashes")["known_answers_from_reference_tests"]
    assert oracle.fmix32(0x41424344, 0xffffeeee) == kat["fmix32(0x41424344, seed 0xffffeeee)"]
    assert oracle.fmix64(0x41424344, 0xffffeeee) == kat["fmix64(0x41424344, seed 0xffffeeee)"]
    assert oracle.murmur3_32(kbytes(0x41424344, 4), 0xffffeeee) == kat["murmur3_32(0x41424344, seed 0xffffeeee)"]
    assert oracle.xxh32(kbytes(123456789, 4), 0) == kat["xxh32_u32(123456789, seed 0)"]
    assert oracle.xxh32(kbytes(42, 4), 0) == kat["xxh32_u32(42, seed 0)"]
    for k, s, name in [(0, 0, "xxh64_u32(0, seed 0)"), (0, 42, "xxh64_u32(0, seed 42)"),
                       (42, 0, "xxh64_u32(42, seed 0)"), (123456789, 0, "xxh64_u32(123456789, seed 0)")]:
        assert oracle.xxh64(kbytes(k, 4), s) == kat[name]
    for k, s, name in [(0, 0, "xxh64_u64(0, seed 0)"), (0, 42, "xxh64_u64(0, seed 42)"),
                       (42, 0, "xxh64_u64(42, seed 0)"), (123456789, 0, "xxh64_u64(123456789, seed 0)")]:
        assert oracle.xxh64(kbytes(k, 8), s) == kat[name]


def test_hash_vectors_match_reference_headers():
    g = load("hashes")
    for r in g["vectors"]:
        kb, k, s = r["key_bytes"], r["key"], r["seed"]
        b = kbytes(k, kb)
        assert oracle.xxh32(b, s) == r["xxh32"]
        assert oracle.murmur3_32(b, s) == r["murmur3_32"]
        fm = oracle.fmix32(k, s) if kb == 4 else oracle.fmix64(k, s)
        assert fm == r["fmix"]
        assert oracle.xxh64(b, s) == r["xxh64"]
    for r in g["xxh64_i64"]:
        assert oracle.xxh64(kbytes(r["key"] & (2**64 - 1), 8), r["seed"]) == r["h"]
    for r in g["xxh64_f32"]:
        assert oracle.xxh64(kbytes(r["bits"], 4), r["seed"]) == r["h"]


def test_two_byte_key_hashes_match_reference_headers():
    """int16/uint16/fp16 keys hash their two bytes: XXH32 and XXH64 through their
    single-byte tail steps, MurmurHash3 through its 2-byte tail (reference headers)."""
    for r in load("hashes")["vectors16"]:
        b = kbytes(r["key"], 2)
        assert oracle.xxh32(b, r["seed"]) == r["xxh32"]
        assert oracle.murmur3_32(b, r["seed"]) == r["murmur3_32"]
        assert oracle.xxh64(b, r["seed"]) == r["xxh64"]


def test_float_key_comparison_matches_reference():
    """EqualTo on fp16 / float / double bit patterns (the reference's EqualWrapper
    compiled here): -0 equals +0, NaN equals nothing.  The sentinel test is
    bitwise for floating-point types (utility/traits.h:27-28); the host probe
    stands in for fp16_t with _Float16, which this C++ library does not classify
    as floating point, so its sentinel rows fall back to == and are not pinned."""
    rows = load("keys")["float_key_comparisons"]
    assert len(rows) == 3 * 144
    for r in rows:
        assert oracle.key_equal(oracle.KEY_FLOAT, r["key_bytes"], r["a"], r["b"]) == bool(r["equal"]), r
        if r["key_bytes"] != 2:
            assert bool(r["sentinel"]) == (r["a"] == r["b"]), r
        assert oracle.key_equal(oracle.KEY_INT, r["key_bytes"], r["a"], r["b"]) == (r["a"] == r["b"])


def test_prime_table_rule_reproduces_reference_table():
    g = load("capacity")
    t = oracle.prime_table().astype(np.int64)
    assert len(t) == g["prime_count"]
    assert hashlib.sha256(t.tobytes()).hexdigest() == g["prime_sha256_le_int64"]
    assert t[:40].tolist() == g["prime_first"]
    assert t[-5:].tolist() == g["prime_last"]


def test_capacity_matches_reference():
    g = load("capacity")
    for row in g["tables"]:
        b, dh = row["bucket_size"], row["double_hashing"]
        probing = oracle.PROBE_DOUBLE if dh else oracle.PROBE_LINEAR
        got = [oracle.valid_capacity(r, b, probing) for r in g["requests"]]
        assert got == row["capacities"], (b, dh)
    assert g["beyond_table_returns_error"] == [0]
    last = int(g["prime_last"][-1])
    assert oracle.valid_capacity(last * 5 + 6, 5, oracle.PROBE_DOUBLE) == 0


def test_probe_walks_match_reference():
    import ctypes as C
    L = oracle.lib()
    L.orc_make_iter.restype = None  # not used directly; walk through the Python loop below
    for r in load("probing")["walks"]:
        kb, b, dh, hk, cap, k = r["key_bytes"], r["bucket_size"], r["double_hashing"], r["hash"], r["capacity"], r["key"]
        nb = cap // b
        h1 = oracle.probe_hash(hk, k, kb, 0)
        idx = (h1 % nb) * b
        step = ((oracle.probe_hash(hk, k, kb, 1) % (nb - 1)) + 1) * b if dh else b
        walk = []
        for _ in range(12):
            walk.append(idx)
            rem = cap - step
            idx = idx - rem if idx >= rem else idx + step
        assert walk == r["walk"], r


def test_bloom_policies_match_reference():
    """Non-default BloomFilterPolicy<Key, xxhash_64, uint32_t, WordsPerBlock, PatternBits>:
    block index and every word pattern of the reference's own template, and the
    oracle's add/contains on them (the 64-entry salt table is pinned here)."""
    rows = load("bloom")["policies"]
    assert {(r["words_per_block"], r["pattern_bits"]) for r in rows} >= {(1, 32), (2, 64), (8, 16), (16, 48), (32, 64)}
    for r in rows:
        wpb, pbits, kb, nb, seed, k = (r["words_per_block"], r["pattern_bits"], r["key_bytes"], r["num_blocks"],
                                       r["seed"], r["key"])
        assert oracle.bloom_policy_valid(wpb, pbits)
        h = oracle.xxh64(kbytes(k, kb), seed)
        assert ((h >> 32) * (nb & 0xffffffff)) >> 32 == r["block"]
        assert oracle.bloom_word_patterns(wpb, pbits, h & 0xffffffff) == r["patterns"]
        if nb <= 257:
            keys = np.array([k], dtype=np.uint32 if kb == 4 else np.uint64)
            words = np.zeros(wpb * nb, dtype=np.uint32)
            oracle.bloom_add(words, nb, keys, seed, wpb, pbits)
            blk = r["block"]
            assert words[blk * wpb:(blk + 1) * wpb].tolist() == r["patterns"]
            assert oracle.bloom_contains(words, nb, keys, seed, 1, wpb, pbits).tolist() == [1]
    for bad in [(3, 3), (64, 64), (8, 4), (8, 12), (4, 80), (1, 33)]:
        assert not oracle.bloom_policy_valid(*bad)


def test_bloom_locate_matches_reference():
    salts = [0x47b6137b, 0x44974d91, 0x8824ad5b, 0xa2b7289d, 0x705495c7, 0x2df1424b, 0x9efc4947, 0x5c6bfb31]
    for r in load("bloom")["locate"]:
        kb, nb, seed, k = r["key_bytes"], r["num_blocks"], r["seed"], r["key"]
        dt = np.uint32 if kb == 4 else np.uint64
        keys = np.array([k], dtype=dt)
        words = np.zeros(8 * nb, dtype=np.uint32) if nb <= 1024 else None
        if words is not None:
            oracle.bloom_add(words, nb, keys, seed)
            blk = r["block"]
            assert words[blk * 8: blk * 8 + 8].tolist() == r["patterns"]
            assert int(words.astype(bool).sum()) == 8
            assert oracle.bloom_contains(words, nb, keys, seed).tolist() == [1]
        h = oracle.xxh64(kbytes(k, kb), seed)
        assert ((h >> 32) * (nb & 0xffffffff)) >> 32 == r["block"]
        lower = h & 0xffffffff
        assert [1 << (((s * lower) & 0xffffffff) >> 27) for s in salts] == r["patterns"]


def test_oracle_open_addressing_against_dict_golden():
    """Unique keys: Find/Contains equal a std::unordered_map-style golden
    (tests/common/golden.h); duplicate inserts fail; InsertAndFind first wins."""
    rng = np.random.default_rng(7)
    for kdt, vdt, b, probing, hk in [(np.int32, np.int32, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32),
                                     (np.int64, np.int64, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32),
                                     (np.int64, np.int64, 1, oracle.PROBE_LINEAR, oracle.HASH_MURMUR3_32),
                                     (np.int32, None, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)]:
        cap = oracle.valid_capacity(4000, b, probing)
        t = oracle.Table(kdt, vdt, cap, b, probing, hk)
        keys = rng.choice(np.arange(1, 100000), size=2000, replace=False).astype(kdt)
        vals = (keys.astype(np.int64) * 3 + 1).astype(vdt) if vdt is not None else None
        assert t.insert(keys, vals) == 0
        assert t.insert(keys[:100], vals[:100] if vals is not None else None) == 100
        q = np.concatenate([keys[:500], rng.integers(200000, 300000, size=500).astype(kdt)])
        out, win = t.find(q)
        exp = (q.astype(np.int64) * 3 + 1) if vdt is not None else q.astype(np.int64)
        assert (out[:500].astype(np.int64) == exp[:500]).all()
        assert (out[500:].astype(np.int64) == -1).all()
        c, _ = t.contains(q)
        assert c.tolist() == [1] * 500 + [0] * 500
        assert (win >= 1).all()
        # empty key is never inserted
        assert t.insert(np.array([-1], dtype=kdt), np.array([5], dtype=vdt) if vdt is not None else None) == 1
    t = oracle.Table(np.int64, np.int64, oracle.valid_capacity(100, 5, oracle.PROBE_DOUBLE))
    f, ins = t.insert_and_find(np.array([5, 6, 5, -1], np.int64), np.array([50, 60, 51, 9], np.int64))
    assert f.tolist() == [50, 60, 50, -1] and ins.tolist() == [1, 1, 0, 0]


def test_oracle_hll_registers_rule():
    """GoldenAdd (tests/hyperloglog/add_test.cpp:321-334): rank counts leading zeros of the tail."""
    rng = np.random.default_rng(3)
    keys = rng.integers(-2**63, 2**63 - 1, size=5000, dtype=np.int64)
    for p in (13, 16, 18):
        reg = np.zeros(1 << p, np.uint8)
        oracle.hll_add(reg, p, keys)
        ref = np.zeros(1 << p, np.uint8)
        for k in keys.tolist():
            h = oracle.xxh64(kbytes(k & (2**64 - 1), 8), 0)
            idx = h >> (64 - p)
            tail = ((h << p) & (2**64 - 1)) | (1 << (p - 1))
            rank = 1
            while not (tail >> 63) & 1:
                rank += 1
                tail = (tail << 1) & (2**64 - 1)
            ref[idx] = max(ref[idx], rank)
        assert (reg == ref).all()
        assert reg.max() <= 65 - p


def test_roaring_oracle_matches_reference():
    """The Roaring oracle (oracle/roaring.py) against the reference's own parser
    and membership query (roaring_bitmap_ref.h, detail/roaring_bitmap/format.h,
    compiled on the host by tests/golden/make_golden.py): the serializer
    reproduces the recorded bytes and the set-based Contains equals the
    reference's answers on every query."""
    from oracle.roaring import contains, golden_cases
    rows = {r["name"]: r for r in load("roaring")["bitmaps"]}
    for name, key64, elements, data, queries, valid in golden_cases():
        r = rows[name]
        assert r["hex"] == data.hex(), name
        assert r["valid"] == valid and r["key64"] == key64, name
        assert r["queries"] == [int(x) for x in queries], name
        if valid:
            assert r["num_keys"] == len(np.unique(elements)) and r["size_bytes"] == len(data), name
            assert contains(elements, queries).astype(int).tolist() == r["contains"], name
