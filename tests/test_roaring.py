"""RoaringBitmap over the portable serialization, against the reference's own
parser and membership query recorded in tests/golden/roaring.json (see
tests/golden/make_golden.py) and the oracle (oracle/roaring.py).

CPU: the library's host parse (b2co_roaring_parse) accepts and measures every
valid case exactly like the reference and rejects every malformed one.
GPU: Contains equals the reference's answers on the recorded queries, and the
oracle's on large random bitmaps of every container kind (mirrors the
reference's tests/roaring_bitmap/contains_test.cpp)."""
import json
import os

import numpy as np
import pytest

from helpers import dev
from oracle.roaring import contains, serialize32, serialize64

GOLD = os.path.join(os.path.dirname(__file__), "golden", "roaring.json")


def rows():
    with open(GOLD) as f:
        return json.load(f)["bitmaps"]


def test_parse_matches_reference():
    import b2co
    for r in rows():
        data = bytes.fromhex(r["hex"])
        kb = 8 if r["key64"] else 4
        if r["valid"]:
            assert b2co.roaring_parse(data, kb) == (r["num_keys"], r["size_bytes"]), r["name"]
            assert b2co.roaring_parse(data, kb, bounded=False) == (r["num_keys"], r["size_bytes"]), r["name"]
        else:
            with pytest.raises(b2co.InvalidArgument):
                b2co.roaring_parse(data, kb)
    with pytest.raises(b2co.InvalidArgument):
        b2co.roaring_parse(b"", 4)  # empty input is truncated


@pytest.mark.gpu
def test_contains_matches_reference_answers():
    import b2co
    import torch
    for r in rows():
        if not r["valid"]:
            continue
        kb = 8 if r["key64"] else 4
        data = bytes.fromhex(r["hex"])
        bm = b2co.RoaringBitmap(data, kb)
        assert bm.Size() == r["num_keys"] and bm.SizeBytes() == r["size_bytes"]
        assert bm.Empty() == (r["num_keys"] == 0)
        assert bm.bytes() == data
        q = np.array(r["queries"], dtype=np.uint64).astype(np.uint32 if kb == 4 else np.uint64)
        qd = dev(q.view(np.int32 if kb == 4 else np.int64))
        out = torch.empty(len(q), dtype=torch.uint8, device="cuda")
        bm.Contains(qd, out)
        assert out.cpu().numpy().tolist() == r["contains"], r["name"]


@pytest.mark.gpu
@pytest.mark.parametrize("run_mode", ["none", "auto", "all"])
@pytest.mark.parametrize("key64", [False, True])
def test_contains_random_bitmaps(run_mode, key64):
    import b2co
    import torch
    rng = np.random.default_rng({"none": 1, "auto": 2, "all": 3}[run_mode] + 10 * int(key64))
    parts = [rng.integers(0, 1 << 24, size=200000),                        # sparse arrays
             (40 << 16) + rng.integers(0, 65536, size=20000),              # bitsets
             (90 << 16) + np.arange(0, 60000), (91 << 16) + np.arange(0, 65536, 3)]  # runs / stripes
    if key64:
        hi = np.array([0, 5, 1 << 20, 2**32 - 1], dtype=np.uint64)
        elems = np.concatenate([(hi[i % 4] << np.uint64(32)) + p.astype(np.uint64) for i, p in enumerate(parts)])
        data = serialize64(elems, run_mode)
        top = 2**64 - 1
    else:
        elems = np.concatenate(parts).astype(np.uint64)
        data = serialize32(elems, run_mode)
        top = 2**32 - 1
    bm = b2co.RoaringBitmap(data, 8 if key64 else 4)
    assert bm.Size() == len(np.unique(elems))
    e = np.unique(elems)
    q = np.concatenate([e[rng.integers(0, len(e), size=300000)], e[rng.integers(0, len(e), size=50000)] + np.uint64(1),
                        rng.integers(0, top, size=300000, dtype=np.uint64, endpoint=True)])
    q = q & np.uint64(top)
    qd = dev(q.astype(np.uint32).view(np.int32) if not key64 else q.view(np.int64))
    out = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    bm.ContainsAsync(qd, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), contains(elems, q).astype(np.uint8))


@pytest.mark.gpu
def test_contains_edge_arguments():
    import b2co
    import torch
    bm = b2co.RoaringBitmap(serialize32([1, 2, 3]), 4)
    bm.Contains(None, None, n=0)  # zero keys: null buffers accepted
    with pytest.raises(b2co.InvalidArgument):
        bm.Contains(None, torch.empty(4, dtype=torch.uint8, device="cuda"), n=4)
    with pytest.raises(b2co.InvalidArgument):
        b2co.RoaringBitmap(b"\x39\x30\x00\x00", 4)  # truncated after the cookie
