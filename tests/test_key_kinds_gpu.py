"""GPU parity for 2-byte keys and payloads and for floating-point keys, through
the C ABI, against the oracle.

The reference instantiates its containers with fp16_t, int16_t and uint16_t
keys and 2-byte payloads (tests/static_set/insert_test.cpp:41-42,
tests/static_map/insert_or_assign_test.cpp:45-46, for_each_test.cpp:70-71)
and with float keys (tests/static_map/find_test.cpp:78-80,
clear_test.cpp:45-46).  Floating-point keys match with == (equal_wrapper.h:
30-33): -0.0 equals +0.0 and a NaN equals nothing, while sentinels compare
bitwise and hashes read the key's bytes.  A 2-byte slot is claimed with a
16-bit compare-and-swap (the narrow CAS of open_addressing_ref_impl.h:
187-199).

Lookups on floating-point tables are compared with the oracle over a host
copy of the device table: whether a -0.0 query reaches a stored +0.0 depends
on where concurrent inserts placed the other keys, so the oracle answers on
the very same slots.  Stored pair sets (as bit patterns) are compared with the
oracle's own sequential build."""
import numpy as np
import pytest

import oracle
from helpers import dev

pytestmark = pytest.mark.gpu

SCHEMES = [
    (5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32),
    (1, oracle.PROBE_LINEAR, oracle.HASH_MURMUR3_32),
    (5, oracle.PROBE_LINEAR, oracle.HASH_MURMUR3_32),
    (4, oracle.PROBE_DOUBLE, oracle.HASH_XXH64),
]

# (key dtype, payload dtype or None) as numpy dtypes
LAYOUTS = [
    (np.int16, None), (np.uint16, np.uint16), (np.int16, np.int16),
    (np.float16, None), (np.float16, np.float16),
    (np.float32, None), (np.float32, np.float32), (np.float32, np.int64),
    (np.float64, None), (np.float64, np.float64), (np.float64, np.int32),
]


def _torch(dt):
    import torch
    return {np.int16: torch.int16, np.uint16: torch.uint16, np.float16: torch.float16, np.float32: torch.float32,
            np.float64: torch.float64, np.int32: torch.int32, np.int64: torch.int64}[np.dtype(dt).type]


def _ubits(a):
    return a.view({2: np.uint16, 4: np.uint32, 8: np.uint64}[a.dtype.itemsize])


def _keys(rng, kdt, n):
    """n keys, distinct by the key's == (so no +0.0 together with -0.0), never
    the -1 sentinel; floating-point keys include a few NaNs (which never match,
    so each NaN insert takes a slot of its own)."""
    kdt = np.dtype(kdt)
    if kdt.kind in "iu":
        pool = np.arange(0, 30000, dtype=np.int64) if kdt.itemsize == 2 else None
        k = rng.choice(pool, size=n, replace=False) if pool is not None else None
        return k.astype(kdt)
    if kdt.itemsize == 2:
        bits = rng.choice(np.arange(0, 0x7c00, dtype=np.uint16), size=n, replace=False)  # finite non-negatives
        sign = rng.integers(0, 2, size=n).astype(np.uint16) << 15
        bits = bits | sign
        k = bits.view(np.float16)
    else:
        k = (rng.standard_normal(int(n * 1.2)) * 1000).astype(kdt)
        k = np.unique(k)[:n]
        rng.shuffle(k)
    # +0.0 must not meet -0.0 in one set: keep +0.0 only
    zero = (k == 0)
    k = np.where(zero, np.zeros(1, kdt), k).astype(kdt)
    _, first = np.unique(_ubits(k.copy()), return_index=True)
    k = k[np.sort(first)]
    k = k[k != -1]
    nan = np.full(3, np.nan, dtype=kdt)
    return np.concatenate([k[: n - 3], nan]).astype(kdt)


def _table(kdt, vdt, scheme, capacity):
    import b2co
    b, probing, hk = scheme
    if vdt is None:
        return b2co.StaticSet(capacity, -1, key_dtype=_torch(kdt), bucket_size=b, probing=probing, hash_kind=hk)
    return b2co.StaticMap(capacity, -1, -1, key_dtype=_torch(kdt), value_dtype=_torch(vdt), bucket_size=b,
                          probing=probing, hash_kind=hk)


def _pairs(keys, vals):
    import b2co
    k = dev(keys)
    return k if vals is None else b2co.pack_pairs(k, dev(vals))


def _vals(rng, vdt, n):
    if vdt is None:
        return None
    vdt = np.dtype(vdt)
    if vdt.kind == "f":
        return (rng.standard_normal(n) * 100).astype(vdt)
    hi = 30000 if vdt.itemsize == 2 else 2**30
    return rng.integers(0, hi, size=n).astype(vdt)


def _out(kdt, vdt, n):
    import torch
    return torch.empty(n, dtype=_torch(vdt if vdt is not None else kdt), device="cuda")


def _queries(rng, keys, kdt, n_miss):
    kdt = np.dtype(kdt)
    miss = _keys(np.random.default_rng(rng.integers(1 << 30)), kdt, n_miss)
    extra = [keys[:200], miss]
    if kdt.kind == "f":  # signed zeros, NaN, infinities, the sentinel
        extra.append(np.array([0.0, -0.0, np.nan, np.inf, -np.inf, -1.0], dtype=kdt))
    else:
        extra.append(np.array([-1 if kdt.kind == "i" else 65535], dtype=kdt))
    q = np.concatenate([keys] + extra).astype(kdt)
    rng.shuffle(q)
    return q


@pytest.mark.parametrize("layout", LAYOUTS, ids=lambda l: f"{np.dtype(l[0]).name}-{l[1] and np.dtype(l[1]).name}")
@pytest.mark.parametrize("scheme", SCHEMES, ids=lambda s: f"b{s[0]}p{s[1]}h{s[2]}")
def test_insert_find_contains_stored_set(layout, scheme):
    import torch
    kdt, vdt = layout
    rng = np.random.default_rng(7 + np.dtype(kdt).itemsize + scheme[0])
    n = 6000
    keys = _keys(rng, kdt, n)
    vals = _vals(rng, vdt, len(keys))
    t = _table(kdt, vdt, scheme, 2 * len(keys))
    o = oracle.Table(kdt, vdt, t.Capacity(), *scheme)
    assert t.Capacity() == oracle.valid_capacity(2 * len(keys), scheme[0], scheme[1])
    assert t.Insert(_pairs(keys, vals)) == o.insert(keys, vals) == 0
    d = oracle.Table(kdt, vdt, t.Capacity(), *scheme)
    d.load_slots(t.dump_slots())
    assert np.array_equal(d.pairs(), o.pairs())

    q = _queries(rng, keys, kdt, 2000)
    out = _out(kdt, vdt, len(q))
    t.Find(dev(q), out)
    exp, _ = d.find(q)
    assert np.array_equal(_ubits(out.cpu().numpy()), _ubits(exp))
    flags = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    t.Contains(dev(q), flags)
    exp_c, _ = d.contains(q)
    assert np.array_equal(flags.cpu().numpy(), exp_c)
    if np.dtype(kdt).kind == "f":
        assert not exp_c[np.isnan(q)].any()  # NaN never matches
    # the same keys again: every one is a duplicate except the NaNs, which take new slots
    again = t.Insert(_pairs(keys, vals))
    assert again == o.insert(keys, vals)
    d.load_slots(t.dump_slots())
    assert np.array_equal(d.pairs(), o.pairs())


@pytest.mark.parametrize("layout", LAYOUTS, ids=lambda l: f"{np.dtype(l[0]).name}-{l[1] and np.dtype(l[1]).name}")
def test_insert_and_find_first_wins_and_assign(layout):
    import b2co
    import torch
    kdt, vdt = layout
    scheme = SCHEMES[0]
    rng = np.random.default_rng(99 + np.dtype(kdt).itemsize)
    keys = _keys(rng, kdt, 5000)
    finite = keys[~np.isnan(keys)] if np.dtype(kdt).kind == "f" else keys
    dups = rng.choice(finite, size=1500)
    stream = np.concatenate([keys, dups]).astype(kdt)
    rng.shuffle(stream)
    vals = _vals(rng, vdt, len(stream))
    t = _table(kdt, vdt, scheme, 2 * len(stream))
    o = oracle.Table(kdt, vdt, t.Capacity(), *scheme)
    found = _out(kdt, vdt, len(stream))
    ins = torch.empty(len(stream), dtype=torch.uint8, device="cuda")
    t.InsertAndFind(_pairs(stream, vals), found, ins, mode=b2co.IAF_FIRST_WINS)
    ef, ei = o.insert_and_find(stream, vals)
    assert np.array_equal(ins.cpu().numpy(), ei)
    assert np.array_equal(_ubits(found.cpu().numpy()), _ubits(ef))
    d = oracle.Table(kdt, vdt, t.Capacity(), *scheme)
    d.load_slots(t.dump_slots())
    assert np.array_equal(d.pairs(), o.pairs())
    if vdt is not None:
        nv = _vals(rng, vdt, len(finite))
        failed, assigned = t.InsertOrAssign(_pairs(finite, nv), with_assigned=True)
        of, oa = o.insert_or_assign(finite, nv)
        assert (failed, assigned) == (of, oa)
        d.load_slots(t.dump_slots())
        assert np.array_equal(d.pairs(), o.pairs())


def test_signed_zero_and_nan_semantics():
    """+0.0 stored, -0.0 looked up in the bucket where +0.0 sits: found by ==.
    A NaN key is inserted every time and never found; the bitwise sentinel
    (-1.0) is never inserted."""
    for kdt in (np.float16, np.float32, np.float64):
        # one bucket of 8 slots under linear probing: every key scans the same window
        t = _table(kdt, kdt, (8, oracle.PROBE_LINEAR, oracle.HASH_MURMUR3_32), 8)
        o = oracle.Table(kdt, kdt, t.Capacity(), 8, oracle.PROBE_LINEAR, oracle.HASH_MURMUR3_32)
        keys = np.array([0.0, 1.5, np.nan, -1.0], dtype=kdt)
        vals = np.array([10, 20, 30, 40], dtype=kdt)
        assert t.Insert(_pairs(keys, vals)) == o.insert(keys, vals) == 1  # the sentinel fails
        q = np.array([-0.0, 0.0, 1.5, np.nan, -1.0, 2.0], dtype=kdt)
        out = _out(kdt, kdt, len(q))
        t.Find(dev(q), out)
        got = out.cpu().numpy()
        exp, _ = o.find(q)
        assert np.array_equal(_ubits(got), _ubits(exp))
        assert got[0] == 10 and got[1] == 10 and got[2] == 20 and got[3] == -1 and got[4] == -1
        # a second NaN insert takes another slot; -0.0 is a duplicate of +0.0
        more = np.array([np.nan, -0.0], dtype=kdt)
        assert t.Insert(_pairs(more, np.array([50, 60], dtype=kdt))) == o.insert(more, np.array([50, 60], dtype=kdt))
        d = oracle.Table(kdt, kdt, t.Capacity(), 8, oracle.PROBE_LINEAR, oracle.HASH_MURMUR3_32)
        d.load_slots(t.dump_slots())
        assert np.array_equal(d.pairs(), o.pairs())
        assert int(np.isnan(d.slot_keys_values()[0]).sum()) == 2


def test_layout_and_hash_errors():
    import b2co
    import torch
    with pytest.raises(b2co.InvalidArgument):  # Fmix takes 4- or 8-byte keys (utils.h:42-66)
        b2co.StaticSet(100, -1, key_dtype=torch.int16, hash_kind=b2co.HASH_FMIX)
    with pytest.raises(b2co.InvalidArgument):  # a 2-byte payload needs a 2-byte key
        b2co.StaticMap(100, -1, -1, key_dtype=torch.int32, value_dtype=torch.int16)
