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
