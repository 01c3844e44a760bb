"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs only where the reference project is mounted: it
builds oracle/ref_probe (the reference's own host-compilable headers compiled
in place, outputs into oracle/_ref/) and records their outputs as plain
numbers.  The fixtures pin the oracle and the product; nothing here runs on
the GPU box.

    python tests/golden/make_golden.py --ref <checkout of the reference project>

(--ref defaults to the B2CO_REFERENCE environment variable, else to a
`reference` directory beside this repository.)
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def load_probe(ref: str):
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle", "ref_probe"), f"REF={ref}"], check=True)
    L = C.CDLL(os.path.join(REPO, "oracle", "_ref", "libref_probe.so"))
    u32, u64, i32, i64, dbl = C.c_uint32, C.c_uint64, C.c_int, C.c_int64, C.c_double
    sig = {
        "ref_xxh32_u32": (u32, [u32, u32]), "ref_xxh32_u64": (u32, [u64, u32]),
        "ref_xxh64_u32": (u64, [u32, u64]), "ref_xxh64_u64": (u64, [u64, u64]),
        "ref_xxh64_i64": (u64, [i64, u64]), "ref_xxh64_f32": (u64, [C.c_float, u64]),
        "ref_murmur3_u32": (u32, [u32, u32]), "ref_murmur3_u64": (u32, [u64, u32]),
        "ref_xxh32_u16": (u32, [C.c_uint16, u32]), "ref_murmur3_u16": (u32, [C.c_uint16, u32]),
        "ref_xxh64_u16": (u64, [C.c_uint16, u64]),
        "ref_equal_f16": (i32, [C.c_uint16, C.c_uint16, i32]), "ref_equal_f32": (i32, [u32, u32, i32]),
        "ref_equal_f64": (i32, [u64, u64, i32]),
        "ref_fmix32": (u32, [u32, u32]), "ref_fmix64": (u64, [u64, u64]),
        "ref_prime_count": (u64, []), "ref_prime_at": (i64, [u64]),
        "ref_valid_capacity": (u64, [u64, i32, i32]),
        "ref_probe_walk": (None, [i32, i32, i32, i32, u64, u32, u32, C.c_void_p]),
        "ref_bloom_locate": (None, [i32, u64, u64, u64, C.c_void_p, C.c_void_p]),
        "ref_bloom_locate_policy": (i32, [i32, u64, u64, u64, u32, u32, C.c_void_p, C.c_void_p]),
        "ref_roaring": (i32, [i32, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ref_hll_finalize": (u64, [i32, dbl, i32]),
        "ref_hll_points": (i32, [i32]), "ref_hll_raw": (dbl, [i32, i32]),
        "ref_hll_bias": (dbl, [i32, i32]), "ref_hll_threshold": (dbl, [i32]),
    }
    for n, (r, a) in sig.items():
        f = getattr(L, n)
        f.restype, f.argtypes = r, a
    return L


def edge_keys(rng, nbytes):
    m = (1 << (8 * nbytes)) - 1
    base = [0, 1, 2, 42, 123456789, 0x41424344, m, m - 1, m >> 1, (m >> 1) + 1, 0xdeadbeef & m]
    return base + [int(x) for x in rng.integers(0, m, size=48, dtype=np.uint64, endpoint=True)]


def hashes(L, rng):
    out = {"known_answers_from_reference_tests": {
        # tests/utility/hash_test.cpp:17-46
        "fmix32(0x41424344, seed 0xffffeeee)": 0x570df661,
        "fmix64(0x41424344, seed 0xffffeeee)": 0x5ee45a8eb612f708,
        "murmur3_32(0x41424344, seed 0xffffeeee)": 0xd6bdbbb4,
        "xxh32_u32(123456789, seed 0)": 0xb20a85ee,
        "xxh32_u32(42, seed 0)": 0x454235d1,
        # tests/utility/xxhash64_test.cpp:88-98
        "xxh64_u32(0, seed 0)": 4246796580750024372, "xxh64_u32(0, seed 42)": 3614696996920510707,
        "xxh64_u32(42, seed 0)": 15516826743637085169, "xxh64_u32(123456789, seed 0)": 9462334144942111946,
        "xxh64_u64(0, seed 0)": 3803688792395291579, "xxh64_u64(0, seed 42)": 13194218611613725804,
        "xxh64_u64(42, seed 0)": 13066772586158965587, "xxh64_u64(123456789, seed 0)": 14662639848940634189,
    }}
    seeds32 = [0, 1, 42, 0xffffeeee]
    rows = []
    for k in edge_keys(rng, 4):
        for s in seeds32:
            rows.append({"key_bytes": 4, "key": k, "seed": s,
                         "xxh32": L.ref_xxh32_u32(k, s), "murmur3_32": L.ref_murmur3_u32(k, s),
                         "fmix": L.ref_fmix32(k, s), "xxh64": L.ref_xxh64_u32(k, s)})
    for k in edge_keys(rng, 8):
        for s in seeds32:
            rows.append({"key_bytes": 8, "key": k, "seed": s,
                         "xxh32": L.ref_xxh32_u64(k, s), "murmur3_32": L.ref_murmur3_u64(k, s),
                         "fmix": L.ref_fmix64(k, s), "xxh64": L.ref_xxh64_u64(k, s)})
    out["vectors"] = rows
    # signed and float keys hash their object representation (xxhash.h:177-183)
    out["xxh64_i64"] = [{"key": int(k), "seed": 0, "h": L.ref_xxh64_i64(int(k), 0)}
                        for k in [-1, -2, -(1 << 63), (1 << 63) - 1, 0]]
    out["xxh64_f32"] = [{"bits": b, "seed": 0,
                         "h": L.ref_xxh64_f32(np.array([b], np.uint32).view(np.float32)[0].item(), 0)}
                        for b in [0x00000000, 0x80000000, 0x3f800000, 0x7fc00000, 0xff800000]]
    # 2-byte keys (int16/uint16/fp16 hash their two bytes): a fixed sample of the key space
    r16 = np.random.default_rng(16)
    keys16 = sorted(set([0, 1, 2, 0x7fff, 0x8000, 0xffff, 0x3c00, 0xbc00, 0x7c00, 0x7e00]
                        + [int(x) for x in r16.integers(0, 1 << 16, size=200)]))
    out["vectors16"] = [{"key": k, "seed": sd, "xxh32": L.ref_xxh32_u16(k, sd), "murmur3_32": L.ref_murmur3_u16(k, sd),
                         "xxh64": L.ref_xxh64_u16(k, sd)} for k in keys16 for sd in (0, 1, 42)]
    return out


def keys(L, rng):
    """The reference's key comparison on floating-point bit patterns: EqualTo (==)
    and the bitwise sentinel test, for fp16, float and double."""
    specials = {
        2: [0x0000, 0x8000, 0x3c00, 0xbc00, 0x7c00, 0xfc00, 0x7e00, 0x7c01, 0xfe00, 0x0001, 0x8001, 0x7bff],
        4: [0x00000000, 0x80000000, 0x3f800000, 0xbf800000, 0x7f800000, 0xff800000, 0x7fc00000, 0x7f800001,
            0xffc00000, 0x00000001, 0x80000001, 0x7f7fffff],
        8: [0x0, 0x8000000000000000, 0x3ff0000000000000, 0xbff0000000000000, 0x7ff0000000000000,
            0xfff0000000000000, 0x7ff8000000000000, 0x7ff0000000000001, 0xfff8000000000000, 0x1,
            0x8000000000000001, 0x7fefffffffffffff],
    }
    fn = {2: L.ref_equal_f16, 4: L.ref_equal_f32, 8: L.ref_equal_f64}
    rows = []
    for kb, vals in specials.items():
        for a in vals:
            for b in vals:
                rows.append({"key_bytes": kb, "a": a, "b": b, "equal": fn[kb](a, b, 0), "sentinel": fn[kb](a, b, 1)})
    return {"float_key_comparisons": rows}


def capacity(L, rng):
    n = L.ref_prime_count()
    table = np.array([L.ref_prime_at(i) for i in range(n)], dtype=np.int64)
    reqs = list(range(0, 300)) + [2 ** e + d for e in range(9, 33) for d in (-1, 0, 1)]
    reqs += [int(x) for x in rng.integers(300, 2 ** 32, size=300, dtype=np.uint64)]
    reqs += [2_097_152, 268_435_456, 65_536, 2_048, 8_388_608, 16_666_667, 333_333_334]
    rows = []
    for b in (1, 2, 4, 5, 8):
        for dh in (0, 1):
            caps = [L.ref_valid_capacity(r, b, dh) for r in reqs]
            rows.append({"bucket_size": b, "double_hashing": dh, "capacities": caps})
    too_big = [L.ref_valid_capacity(int(table[-1]) * 5 + 6, 5, 1)]
    return {
        "prime_count": int(n),
        "prime_sha256_le_int64": hashlib.sha256(table.tobytes()).hexdigest(),
        "prime_first": table[:40].tolist(), "prime_last": table[-5:].tolist(),
        "prime_sample_index": list(range(0, int(n), 997)),
        "prime_sample": table[::997].tolist(),
        "requests": reqs, "tables": rows, "beyond_table_returns_error": too_big,
    }


def probing(L, rng):
    rows = []
    for kb in (4, 8):
        for b in (1, 5, 8):
            for dh in (0, 1):
                for hk in (0, 1, 2, 3):
                    for cap_req in (40, 1000, 2_097_152):
                        cap = L.ref_valid_capacity(cap_req, b, dh)
                        for k in edge_keys(rng, kb)[:6]:
                            buf = (C.c_uint32 * 12)()
                            L.ref_probe_walk(kb, b, dh, hk, k, cap, 12, buf)
                            rows.append({"key_bytes": kb, "bucket_size": b, "double_hashing": dh, "hash": hk,
                                         "capacity": cap, "key": k, "walk": list(buf)})
    r16 = np.random.default_rng(17)
    for b in (1, 5, 8):
        for dh in (0, 1):
            for hk in (0, 1, 3):  # no Fmix for 2-byte keys
                for cap_req in (40, 1000, 70_000):
                    cap = L.ref_valid_capacity(cap_req, b, dh)
                    for k in [0, 0xffff, 0x8000] + [int(x) for x in r16.integers(0, 1 << 16, size=3)]:
                        buf = (C.c_uint32 * 12)()
                        L.ref_probe_walk(2, b, dh, hk, k, cap, 12, buf)
                        rows.append({"key_bytes": 2, "bucket_size": b, "double_hashing": dh, "hash": hk,
                                     "capacity": cap, "key": k, "walk": list(buf)})
    return {"walks": rows}


def bloom(L, rng):
    rows = []
    for kb in (4, 8):
        for nb in (1, 7, 1024, 1 << 22, (1 << 32) - 1):
            for seed in (0, 42):
                for k in edge_keys(rng, kb)[:20]:
                    blk = C.c_uint32()
                    pat = (C.c_uint32 * 8)()
                    L.ref_bloom_locate(kb, k, nb, seed, C.byref(blk), pat)
                    rows.append({"key_bytes": kb, "num_blocks": nb, "seed": seed, "key": k,
                                 "block": blk.value, "patterns": list(pat)})
    # non-default policies (WordsPerBlock, PatternBits), from the reference's own
    # BloomFilterPolicy template; a separate generator keeps the rows above and
    # the sections after this one unchanged
    prng = np.random.default_rng(4242)
    policy_rows = []
    for wpb, pbits in POLICIES:
        for kb in (4, 8):
            for nb in (1, 257, 1 << 20):
                for seed in (0, 42):
                    for k in edge_keys(prng, kb)[:12]:
                        blk = C.c_uint32()
                        pat = (C.c_uint32 * wpb)()
                        assert L.ref_bloom_locate_policy(kb, k, nb, seed, wpb, pbits, C.byref(blk), pat) == 0
                        policy_rows.append({"words_per_block": wpb, "pattern_bits": pbits, "key_bytes": kb,
                                            "num_blocks": nb, "seed": seed, "key": k, "block": blk.value,
                                            "patterns": list(pat)})
    return {"locate": rows, "policies": policy_rows}


# (WordsPerBlock, PatternBits) of the policy fixtures: every word count the
# policy allows, one and several bits per word, up to the 64-entry salt table.
POLICIES = [(1, 1), (1, 32), (2, 2), (2, 64), (4, 4), (4, 16), (8, 8), (8, 16), (8, 64), (16, 16), (16, 48),
            (32, 32), (32, 64)]


def hll(L, rng):
    tables = {}
    cases = []
    for p in range(13, 19):
        n = L.ref_hll_points(p)
        raw = np.array([L.ref_hll_raw(p, i) for i in range(n)], dtype=np.float64)
        bias = np.array([L.ref_hll_bias(p, i) for i in range(n)], dtype=np.float64)
        tables[str(p)] = {"points": int(n), "threshold": L.ref_hll_threshold(p),
                          "sha256_raw_then_bias_f64le": hashlib.sha256(raw.tobytes() + bias.tobytes()).hexdigest()}
        m = 1 << p
        # synthetic histograms spanning linear counting, the threshold, the
        # bias-interpolation band and the plain-HLL range
        for card in np.unique(np.concatenate([
                np.geomspace(1, 60 * m, 70).astype(np.int64),
                rng.integers(int(2.4 * m), int(5.2 * m), size=40)])):
            reg = np.zeros(m, dtype=np.uint8)
            keys = rng.integers(0, 2 ** 63 - 1, size=int(card), dtype=np.int64)
            # registers from the same rule as HyperLogLogRef::Add via the oracle
            import oracle  # noqa: E402  (repo root on sys.path below)
            oracle.hll_add(reg, p, keys)
            hist = oracle.hll_histogram(reg, p)
            z = float(sum(np.ldexp(float(hist[r]), -r) for r in range(65)))
            cases.append({"precision": p, "hist": hist.tolist(), "z": z, "v": int(hist[0]),
                          "estimate": L.ref_hll_finalize(p, z, int(hist[0]))})
    return {"tables": tables, "finalizer_cases": cases}


def roaring(L, rng):
    """The reference's own portable-format parser and membership query
    (roaring_bitmap_ref.h, detail/roaring_bitmap/format.h) over the oracle's
    deterministic cases: validity, key count, serialized size, Contains."""
    from oracle.roaring import golden_cases
    rows = []
    for name, key64, _, data, queries, valid in golden_cases():
        q = np.ascontiguousarray(queries, dtype=np.uint64)
        out = np.zeros(len(q), dtype=np.uint8)
        nk, sb = C.c_uint64(), C.c_uint64()
        buf = C.create_string_buffer(data, len(data))
        st = L.ref_roaring(int(key64), buf, len(data), q.ctypes.data, len(q), out.ctypes.data, C.byref(nk),
                           C.byref(sb))
        assert (st == 0) == valid, name
        rows.append({"name": name, "key64": bool(key64), "hex": data.hex(), "valid": st == 0,
                     "num_keys": nk.value if st == 0 else None, "size_bytes": sb.value if st == 0 else None,
                     "queries": [int(x) for x in q], "contains": out.tolist() if st == 0 else None})
    return {"bitmaps": rows}


def main():
    import sys
    sys.path.insert(0, REPO)
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("B2CO_REFERENCE")
                    or os.path.join(os.path.dirname(REPO), "reference"))
    args = ap.parse_args()
    if not os.path.isdir(os.path.join(args.ref, "include")):
        ap.error(f"no reference checkout at {args.ref}: name it with --ref or B2CO_REFERENCE")
    L = load_probe(args.ref)
    rng = np.random.default_rng(2026)
    for name, fn in [("hashes", hashes), ("capacity", capacity), ("probing", probing), ("bloom", bloom),
                     ("hll", hll), ("roaring", roaring), ("keys", keys)]:
        data = fn(L, rng)
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(data, f, separators=(",", ":"))
        print(name, os.path.getsize(os.path.join(HERE, f"{name}.json")), "bytes")


if __name__ == "__main__":
    main()
