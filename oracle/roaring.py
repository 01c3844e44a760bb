"""Roaring bitmap oracle: a portable-format serializer and set-based Contains.

TEST INFRASTRUCTURE ONLY, like the rest of ``oracle/``: it builds the
serialized inputs the tests feed to the CUDA RoaringBitmap and answers
Contains from the element set.  The product only parses serialized bitmaps.

The byte format is the published Roaring portable serialization
(RoaringFormatSpec), which the reference consumes
(include/detail/roaring_bitmap/format.h:164-262 for 32-bit keys, :269-318 for
the 64-bit bucketed form):

* cookie 12346 (no run containers): u32 cookie, u32 container count;
  cookie 12347: u16 12347 | (count - 1) << 16, then a bitmap of run
  containers ((count + 7) / 8 bytes);
* per container: u16 high key (strictly increasing), u16 cardinality - 1;
* a u32 offset per container, present unless the bitmap has runs and fewer
  than 4 containers;
* containers: array (cardinality <= 4096 sorted u16), bitset (8 KiB), or run
  (u16 run count, then (start, length - 1) u16 pairs);
* 64-bit: u64 bucket count, then per bucket a u32 high key (strictly
  increasing) followed by a 32-bit portable bitmap of the low halves.
All integers little-endian.
"""
from __future__ import annotations

import struct

import numpy as np


def _runs(values: np.ndarray):
    """(start, length - 1) runs of a sorted unique uint16 array."""
    if len(values) == 0:
        return []
    breaks = np.nonzero(np.diff(values.astype(np.int64)) != 1)[0]
    starts = np.concatenate([[0], breaks + 1])
    ends = np.concatenate([breaks, [len(values) - 1]])
    return [(int(values[s]), int(values[e] - values[s])) for s, e in zip(starts, ends)]


def serialize32(elements, run_mode: str = "auto", force_offsets: bool | None = None) -> bytes:
    """Portable 32-bit serialization of a set of uint32 values.

    run_mode: "none" (no run containers, cookie 12346), "all" (every container
    a run container), or "auto" (a container is a run container when that is
    smaller than its array / bitset form)."""
    vals = np.unique(np.asarray(elements, dtype=np.uint64).astype(np.uint32))
    hi = (vals >> 16).astype(np.uint16)
    keys, starts = np.unique(hi, return_index=True)
    bounds = list(starts) + [len(vals)]
    containers = []
    for i, k in enumerate(keys):
        lo = (vals[bounds[i]:bounds[i + 1]] & 0xFFFF).astype(np.uint16)
        card = len(lo)
        runs = _runs(lo)
        plain_bytes = 2 * card if card <= 4096 else 8192
        run_bytes = 2 + 4 * len(runs)
        is_run = run_mode == "all" or (run_mode == "auto" and run_bytes < plain_bytes)
        if is_run:
            body = struct.pack("<H", len(runs)) + b"".join(struct.pack("<HH", s, l) for s, l in runs)
        elif card <= 4096:
            body = lo.astype("<u2").tobytes()
        else:
            bits = np.zeros(65536, dtype=np.uint8)
            bits[lo] = 1
            body = np.packbits(bits, bitorder="little").tobytes()
        containers.append((int(k), card, is_run, body))
    n = len(containers)
    has_run = any(c[2] for c in containers)
    out = bytearray()
    if has_run:
        out += struct.pack("<I", 12347 | ((n - 1) << 16))
        bitmap = np.zeros((n + 7) // 8 * 8, dtype=np.uint8)
        for i, c in enumerate(containers):
            bitmap[i] = c[2]
        out += np.packbits(bitmap, bitorder="little").tobytes()
    else:
        out += struct.pack("<II", 12346, n)
    for k, card, _, _ in containers:
        out += struct.pack("<HH", k, card - 1)
    with_offsets = (not has_run) or n >= 4
    if force_offsets is not None:
        with_offsets = force_offsets
    header_end = len(out) + (4 * n if with_offsets else 0)
    offsets, pos = [], header_end
    for c in containers:
        offsets.append(pos)
        pos += len(c[3])
    if with_offsets:
        out += b"".join(struct.pack("<I", o) for o in offsets)
    for c in containers:
        out += c[3]
    return bytes(out)


def serialize64(elements, run_mode: str = "auto") -> bytes:
    vals = np.unique(np.asarray(elements, dtype=np.uint64))
    hi = (vals >> np.uint64(32)).astype(np.uint32)
    keys, starts = np.unique(hi, return_index=True)
    bounds = list(starts) + [len(vals)]
    out = bytearray(struct.pack("<Q", len(keys)))
    for i, k in enumerate(keys):
        out += struct.pack("<I", int(k))
        out += serialize32((vals[bounds[i]:bounds[i + 1]] & np.uint64(0xFFFFFFFF)).astype(np.uint32), run_mode)
    return bytes(out)


def _queries(elements, rng, key64: bool, k: int = 300):
    e = np.unique(np.asarray(elements, dtype=np.uint64))
    top = 2**64 - 1 if key64 else 2**32 - 1
    pick = e[rng.integers(0, len(e), size=min(k, len(e)))] if len(e) else np.zeros(0, np.uint64)
    near = np.concatenate([pick + np.uint64(1), np.where(pick > 0, pick - np.uint64(1), pick)]) if len(e) else pick
    rnd = rng.integers(0, top, size=k, dtype=np.uint64, endpoint=True)
    edge = np.array([0, 1, 65535, 65536, top, top - 1], dtype=np.uint64)
    q = np.concatenate([pick, near, rnd, edge])
    return q & np.uint64(top)


def golden_cases():
    """Deterministic (name, key64, elements, serialized bytes, queries, valid)
    cases covering every container kind and header form, 64-bit buckets, and
    malformed inputs; shared by the fixture generator and the tests."""
    rng = np.random.default_rng(20261203)
    cases = []

    def add(name, key64, elements, data, valid=True):
        cases.append((name, key64, np.asarray(elements, dtype=np.uint64), data,
                      _queries(elements, rng, key64), valid))

    add("u32-empty", False, [], serialize32([]))
    acc = [(1 << 16) | 2, (1 << 16) | 4, (1 << 16) | 8]
    add("u32-three-keys", False, acc, serialize32(acc, "none"))
    arr = np.unique(rng.integers(0, 12 << 16, size=900, dtype=np.uint64))
    add("u32-arrays-12-containers", False, arr, serialize32(arr, "none"))
    dense = np.concatenate([(3 << 16) + np.unique(rng.integers(0, 65536, size=9000)),
                            np.unique(rng.integers(5 << 16, 6 << 16, size=40))]).astype(np.uint64)
    add("u32-bitset-and-array", False, dense, serialize32(dense, "none"))
    runs2 = np.concatenate([np.arange(100, 2100), (9 << 16) + np.arange(0, 65536, 2)[:50]]).astype(np.uint64)
    add("u32-runs-no-offsets", False, runs2, serialize32(runs2, "all"))
    mixed = np.concatenate([np.arange(10, 5000),                                      # run (auto)
                            (1 << 16) + np.unique(rng.integers(0, 65536, size=300)),   # array
                            (2 << 16) + np.unique(rng.integers(0, 65536, size=6000)),  # bitset
                            (4 << 16) + np.arange(0, 65536),                           # one full run
                            (7 << 16) + np.array([0, 65535]),                          # array edges
                            (0xFFFF << 16) + np.arange(65000, 65536)]).astype(np.uint64)
    add("u32-mixed-with-runs", False, mixed, serialize32(mixed, "auto"))
    many = np.unique(rng.integers(0, 40 << 16, size=2000, dtype=np.uint64))
    add("u32-runs-all-40-containers", False, many, serialize32(many, "all"))
    b64 = np.concatenate([np.arange(5, 600),
                          (np.uint64(7) << np.uint64(32)) + np.array(acc, dtype=np.uint64),
                          (np.uint64(7) << np.uint64(32)) + (3 << 16) + np.unique(rng.integers(0, 65536, size=5000)),
                          (np.uint64(0xFFFFFFFF) << np.uint64(32)) + np.arange(0, 70000, 7)]).astype(np.uint64)
    add("u64-three-buckets", True, b64, serialize64(b64))
    add("u64-empty", True, [], serialize64([]))
    # malformed inputs the reference's parser rejects
    base = serialize32(dense, "none")
    add("bad-truncated", False, [], base[: len(base) - 100], valid=False)
    add("bad-cookie", False, [], struct.pack("<II", 12345, 0), valid=False)
    swapped = bytearray(serialize32(arr, "none"))
    swapped[8:12], swapped[12:16] = swapped[12:16], swapped[8:12]  # first two container keys out of order
    add("bad-decreasing-keys", False, [], bytes(swapped), valid=False)
    off = bytearray(serialize32(arr, "none"))
    n = struct.unpack_from("<I", off, 4)[0]
    struct.pack_into("<I", off, 8 + 4 * n, 0)  # first container offset inside the header
    add("bad-offset", False, [], bytes(off), valid=False)
    b64bad = bytearray(struct.pack("<Q", 2))
    b64bad += struct.pack("<I", 9) + serialize32([1, 2, 3]) + struct.pack("<I", 4) + serialize32([5])
    add("bad-decreasing-buckets", True, [], bytes(b64bad), valid=False)
    return cases


def contains(elements, queries) -> np.ndarray:
    """1 where the query is in the element set (the Contains result)."""
    s = np.unique(np.asarray(elements, dtype=np.uint64))
    q = np.asarray(queries, dtype=np.uint64)
    pos = np.searchsorted(s, q)
    pos = np.minimum(pos, max(len(s) - 1, 0))
    return (len(s) > 0) & (s[pos] == q) if len(s) else np.zeros(len(q), dtype=bool)
