"""GPU tests for DynamicMap (tests/dynamic_map/*_test.cpp): growth across
submaps, exact dedup against older submaps, fan-out Find/Contains with device
merge, InsertOrAssign, Erase with tombstones, Clear and Reserve -- checked
against a host dictionary golden (tests/common/golden.h)."""
import numpy as np
import pytest

from helpers import dev, miss_keys, unique_keys

pytestmark = pytest.mark.gpu


def pairs(keys, vals):
    import b2co
    return b2co.pack_pairs(dev(keys), dev(vals))


@pytest.mark.parametrize("kb,vb", [(4, 4), (8, 8), (8, 4)])
def test_dynamic_map_growth_find_erase(kb, vb):
    import b2co
    import torch
    kdt = {4: np.int32, 8: np.int64}
    tdt = {4: torch.int32, 8: torch.int64}
    rng = np.random.default_rng(kb * 3 + vb)
    m = b2co.DynamicMap(50000, -1, -1, -2, key_dtype=tdt[kb], value_dtype=tdt[vb])
    gold = {}
    keys = unique_keys(rng, 400000, kb)
    vals = rng.integers(0, 2**30, size=len(keys)).astype(kdt[vb])
    off = 0
    for size in (20000, 60000, 150000, 170000):
        k, v = keys[off:off + size], vals[off:off + size]
        # re-insert some old keys in each batch: exact dedup keeps the first value
        if off:
            k = np.concatenate([k, keys[:1000]])
            v = np.concatenate([v, vals[:1000] + 1])
        got = m.Insert(pairs(k, v))
        new = sum(1 for x in k if int(x) not in gold)
        for x, y in zip(k.tolist(), v.tolist()):
            gold.setdefault(x, y)
        assert got == new
        off += size
    assert m.Size() == len(gold)
    assert m.NumSubmaps() > 1
    q = np.concatenate([keys, miss_keys(rng, 20000, kb)])
    out = torch.empty(len(q), dtype=tdt[vb], device="cuda")
    m.Find(dev(q), out)
    exp = np.array([gold.get(int(x), -1) for x in q], dtype=kdt[vb])
    assert np.array_equal(out.cpu().numpy(), exp)
    c = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    m.Contains(dev(q), c)
    assert np.array_equal(c.cpu().numpy(), (exp != -1).astype(np.uint8) | np.isin(q, list(gold)).astype(np.uint8))

    gone = keys[::7]
    assert m.Erase(dev(gone)) == len(gone)
    for x in gone.tolist():
        gold.pop(x)
    m.Find(dev(q), out)
    exp = np.array([gold.get(int(x), -1) for x in q], dtype=kdt[vb])
    assert np.array_equal(out.cpu().numpy(), exp)
    assert m.Size() == len(gold)

    # InsertOrAssign counts only new keys and overwrites existing payloads everywhere
    upd = np.concatenate([keys[1:50000:3], unique_keys(rng, 5000, kb, lo=2**29 if kb == 4 else 2**61)])
    uv = rng.integers(0, 2**30, size=len(upd)).astype(kdt[vb])
    new = sum(1 for x in upd.tolist() if x not in gold)
    assert m.InsertOrAssign(pairs(upd, uv)) == new
    for x, y in zip(upd.tolist(), uv.tolist()):
        gold[x] = y
    out2 = torch.empty(len(upd), dtype=tdt[vb], device="cuda")
    m.Find(dev(upd), out2)
    assert np.array_equal(out2.cpu().numpy(), uv)

    m.Clear()
    assert m.Size() == 0
    m.Find(dev(q), out)
    assert (out.cpu().numpy() == -1).all()


def test_dynamic_map_reserve_and_append_unique():
    import b2co
    import torch
    rng = np.random.default_rng(5)
    m = b2co.DynamicMap(20000, -1, -1, -2)
    m.Reserve(200000)
    subs = m.NumSubmaps()
    assert subs >= 2
    keys = unique_keys(rng, 100000, 4)
    vals = rng.integers(0, 2**30, size=len(keys)).astype(np.int32)
    assert m.Insert(pairs(keys, vals), mode=b2co.DynamicMap.kAppendUnique) == len(keys)
    out = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    m.Find(dev(keys), out)
    assert np.array_equal(out.cpu().numpy(), vals)
    assert m.Capacity() >= 200000


@pytest.mark.parametrize("kdt,vdt", [(np.int16, np.int16), (np.uint16, np.uint16), (np.float16, np.float16),
                                     (np.float32, np.float32), (np.float64, np.float64), (np.float32, np.int64)],
                         ids=lambda d: np.dtype(d).name)
def test_dynamic_map_two_byte_and_float_keys(kdt, vdt):
    """The reference's DynamicMap tests instantiate (uint16, uint16) and
    (float, float) maps (tests/dynamic_map/*_test.cpp).  Growth over several
    submaps, exact dedup and fan-out Find, checked against a dict; sentinels
    compare by their bits.  (Signed zeros and NaNs follow the probe: their
    cases are checked against the oracle in test_key_kinds_gpu.py.)"""
    import b2co
    import torch
    rng = np.random.default_rng(np.dtype(kdt).itemsize * 7 + np.dtype(vdt).itemsize)
    if np.dtype(kdt).kind == "f":
        pool = rng.uniform(-1000.0, 1000.0, size=60000).astype(kdt)
        pool = np.unique(pool[np.isfinite(pool)])
        pool = pool[(pool != -1.0) & (pool != -2.0) & (pool != 0.0)]
        keys = np.concatenate([np.array([0.0], dtype=kdt), rng.permutation(pool)[:20000]])
    else:
        lo = -30000 if np.dtype(kdt).kind == "i" else 0
        pool = np.arange(lo, lo + 60000, dtype=np.int64)
        pool = pool[(pool != -1) & (pool != -2) & (pool != np.iinfo(kdt).max) & (pool != np.iinfo(kdt).max - 1)]
        keys = rng.permutation(pool)[:20000].astype(kdt)
    if np.dtype(vdt).kind == "f":
        vals = rng.uniform(0.0, 100.0, size=len(keys)).astype(vdt)
    else:
        vals = rng.integers(1, 20000, size=len(keys)).astype(vdt)
    to_t = {np.dtype(np.int16): torch.int16, np.dtype(np.uint16): torch.int16, np.dtype(np.float16): torch.float16,
            np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
            np.dtype(np.int64): torch.int64}
    ek = -1 if np.dtype(kdt).kind != "u" else np.iinfo(kdt).max
    xk = -2 if np.dtype(kdt).kind != "u" else np.iinfo(kdt).max - 1
    m = b2co.DynamicMap(4000, kdt(ek), vdt(-1 if np.dtype(vdt).kind != "u" else 0), kdt(xk),
                        key_dtype=to_t[np.dtype(kdt)], value_dtype=to_t[np.dtype(vdt)])
    empty_v = np.array([-1 if np.dtype(vdt).kind != "u" else 0], dtype=vdt)[0]
    gold = {}
    off = 0
    for size in (3000, 5000, 6000, 6001):
        k, v = keys[off:off + size], vals[off:off + size]
        if off:  # old keys again (dedup keeps the first payload)
            k = np.concatenate([k, keys[:500]])
            v = np.concatenate([v, vals[:500]])
        got = m.Insert(b2co.pack_pairs(dev(k), dev(v)))
        new = 0
        for x, y in zip(k.tolist(), v.tolist()):
            if x not in gold:
                gold[x] = y
                new += 1
        assert got == new
        off += size
    assert m.Size() == len(gold)
    assert m.NumSubmaps() > 1
    misses = np.array([x for x in (pool[-3000:] if np.dtype(kdt).kind == "f" else pool[-3000:].astype(kdt))
                       if x not in gold][:1000], dtype=kdt)
    q = np.concatenate([keys, misses])
    out = torch.empty(len(q), dtype=to_t[np.dtype(vdt)], device="cuda")
    m.Find(dev(q), out)
    exp = np.array([gold.get(x, empty_v) for x in q.tolist()], dtype=vdt)
    assert np.array_equal(out.cpu().numpy().view(np.uint8), exp.view(np.uint8))
    c = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    m.Contains(dev(q), c)
    assert np.array_equal(c.cpu().numpy(), np.array([x in gold for x in q.tolist()], dtype=np.uint8))

