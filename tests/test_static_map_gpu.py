"""GPU parity tests for StaticMap / StaticSet through the C ABI, against the CPU
oracle on the same seeded inputs.  Integer results must be bit-exact; the
stored pair set must be identical (slot order may differ under concurrency).
Mirrors the reference's tests/static_map/*_test.cpp and tests/static_set/*."""
import numpy as np
import pytest

import oracle
from helpers import LAYOUTS, NP_DT, dev, make_pairs, miss_keys, oracle_table, stored_pairs, torch_dt, unique_keys

pytestmark = pytest.mark.gpu

SCHEMES = [  # (bucket size, probing, hash)
    (5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32),
    (1, oracle.PROBE_LINEAR, oracle.HASH_MURMUR3_32),
    (8, oracle.PROBE_DOUBLE, oracle.HASH_MURMUR3_32),
    (2, oracle.PROBE_LINEAR, oracle.HASH_FMIX),
    (4, oracle.PROBE_DOUBLE, oracle.HASH_XXH64),
]


def make_table(kb, vb, b, probing, hk, capacity, erased_key=None):
    import b2co
    import torch
    if vb == 0:
        return b2co.StaticSet(capacity, -1, key_dtype=torch_dt(kb), bucket_size=b, probing=probing, hash_kind=hk,
                              erased_key=erased_key)
    return b2co.StaticMap(capacity, -1, -1, key_dtype=torch_dt(kb), value_dtype=torch_dt(vb), bucket_size=b,
                          probing=probing, hash_kind=hk, erased_key=erased_key)


def values_for(rng, keys, vb):
    if vb == 0:
        return None
    v = rng.integers(0, 2**31 - 2 if vb == 4 else 2**62, size=len(keys), dtype=np.int64)
    return v.astype(NP_DT[vb])


def out_buf(n, kb, vb):
    import torch
    return torch.empty(n, dtype=torch_dt(vb if vb else kb), device="cuda")


@pytest.mark.parametrize("layout", LAYOUTS, ids=lambda l: f"k{l[0]}v{l[1]}")
@pytest.mark.parametrize("scheme", SCHEMES, ids=lambda s: f"b{s[0]}p{s[1]}h{s[2]}")
def test_insert_find_contains_count_parity(layout, scheme):
    import torch
    kb, vb = layout
    b, probing, hk = scheme
    rng = np.random.default_rng(1000 + kb * 10 + vb + b)
    n = 20000
    keys = unique_keys(rng, n + 10000, kb)
    ins, miss = keys[:n], keys[n:]
    vals = values_for(rng, ins, vb)
    t = make_table(kb, vb, b, probing, hk, 2 * n)
    o = oracle_table(t, kb, vb, b, probing, hk)
    assert t.Capacity() == oracle.valid_capacity(2 * n, b, probing)

    pairs = make_pairs(ins, vals)
    assert t.Insert(pairs) == o.insert(ins, vals) == 0
    # re-inserting present keys fails (duplicate), as does the empty key
    assert t.Insert(pairs[:1000]) == o.insert(ins[:1000], None if vals is None else vals[:1000]) == 1000
    got, _ = stored_pairs(t, kb, vb, b, probing, hk)
    assert np.array_equal(got, o.pairs())

    q = np.concatenate([ins[::2], miss, np.array([-1], dtype=NP_DT[kb])])
    rng.shuffle(q)
    qd = dev(q)
    out = out_buf(len(q), kb, vb)
    t.Find(qd, out)
    exp, _ = o.find(q)
    assert np.array_equal(out.cpu().numpy(), exp)
    c = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    t.Contains(qd, c)
    expc, _ = o.contains(q)
    assert np.array_equal(c.cpu().numpy(), expc)
    assert t.Count(qd) == o.count(q) == len(ins[::2])

    stencil = (rng.random(len(q)) < 0.5).astype(np.uint8)
    t.FindIf(qd, dev(stencil), out)
    exp, _ = o.find(q, stencil)
    assert np.array_equal(out.cpu().numpy(), exp)
    t.ContainsIf(qd, dev(stencil), c)
    expc, _ = o.contains(q, stencil)
    assert np.array_equal(c.cpu().numpy(), expc)


@pytest.mark.parametrize("layout", LAYOUTS, ids=lambda l: f"k{l[0]}v{l[1]}")
def test_insert_if_parity(layout):
    kb, vb = layout
    b, probing, hk = SCHEMES[0]
    rng = np.random.default_rng(77)
    keys = unique_keys(rng, 30000, kb)
    vals = values_for(rng, keys, vb)
    stencil = (rng.random(len(keys)) < 0.3).astype(np.uint8)
    t = make_table(kb, vb, b, probing, hk, 50000)
    o = oracle_table(t, kb, vb, b, probing, hk)
    assert t.InsertIf(make_pairs(keys, vals), dev(stencil)) == o.insert(keys, vals, stencil) == 0
    got, _ = stored_pairs(t, kb, vb, b, probing, hk)
    assert np.array_equal(got, o.pairs())
    assert len(got) == int(stencil.sum())


@pytest.mark.parametrize("layout", LAYOUTS, ids=lambda l: f"k{l[0]}v{l[1]}")
@pytest.mark.parametrize("scheme", SCHEMES[:3], ids=lambda s: f"b{s[0]}p{s[1]}h{s[2]}")
def test_insert_and_find_first_wins_matches_sequential(layout, scheme):
    """tests/static_map/insert_and_find_test.cpp: with duplicates in the batch
    and keys already present, first-wins mode equals the sequential golden."""
    import b2co
    import torch
    kb, vb = layout
    b, probing, hk = scheme
    rng = np.random.default_rng(4242 + kb + vb + b)
    base = unique_keys(rng, 40000, kb)
    pre, fresh = base[:5000], base[5000:]
    dups = rng.choice(np.concatenate([fresh[:20000], pre[:2000]]), size=4000)
    keys = np.concatenate([fresh, dups, np.array([-1], dtype=NP_DT[kb])])
    rng.shuffle(keys)
    vals = values_for(rng, keys, vb)
    t = make_table(kb, vb, b, probing, hk, 90000)
    o = oracle_table(t, kb, vb, b, probing, hk)
    pre_vals = values_for(rng, pre, vb)
    assert t.Insert(make_pairs(pre, pre_vals)) == o.insert(pre, pre_vals) == 0

    found = out_buf(len(keys), kb, vb)
    inserted = torch.empty(len(keys), dtype=torch.uint8, device="cuda")
    t.InsertAndFind(make_pairs(keys, vals), found, inserted, mode=b2co.IAF_FIRST_WINS)
    ef, ei = o.insert_and_find(keys, vals)
    assert np.array_equal(inserted.cpu().numpy(), ei)
    assert np.array_equal(found.cpu().numpy(), ef)
    got, _ = stored_pairs(t, kb, vb, b, probing, hk)
    assert np.array_equal(got, o.pairs())


def test_first_wins_batches_on_two_streams_apply_in_call_order():
    """Two asynchronous first-wins batches on different streams share the
    table's scratch: the second waits on the GPU for the first, so the result
    is the two batches applied in call order."""
    import b2co
    import torch
    rng = np.random.default_rng(77)
    keys = unique_keys(rng, 300000, 8)
    a_keys = np.concatenate([keys[:200000], keys[:20000]])
    b_keys = np.concatenate([keys[100000:], keys[150000:170000]])
    rng.shuffle(a_keys)
    rng.shuffle(b_keys)
    a_vals, b_vals = values_for(rng, a_keys, 8), values_for(rng, b_keys, 8)
    t = make_table(8, 8, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, 600000)
    o = oracle_table(t, 8, 8, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    fa, ia = out_buf(len(a_keys), 8, 8), torch.empty(len(a_keys), dtype=torch.uint8, device="cuda")
    fb, ib = out_buf(len(b_keys), 8, 8), torch.empty(len(b_keys), dtype=torch.uint8, device="cuda")
    pa, pb = make_pairs(a_keys, a_vals), make_pairs(b_keys, b_vals)
    torch.cuda.synchronize()
    t.InsertAndFindAsync(pa, fa, ia, stream=s1, mode=b2co.IAF_FIRST_WINS)
    t.InsertAndFindAsync(pb, fb, ib, stream=s2, mode=b2co.IAF_FIRST_WINS)
    torch.cuda.synchronize()
    ef, ei = o.insert_and_find(a_keys, a_vals)
    assert np.array_equal(ia.cpu().numpy(), ei) and np.array_equal(fa.cpu().numpy(), ef)
    ef, ei = o.insert_and_find(b_keys, b_vals)
    assert np.array_equal(ib.cpu().numpy(), ei) and np.array_equal(fb.cpu().numpy(), ef)
    got, _ = stored_pairs(t, 8, 8, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    assert np.array_equal(got, o.pairs())


@pytest.mark.parametrize("layout", LAYOUTS, ids=lambda l: f"k{l[0]}v{l[1]}")
def test_insert_and_find_race_invariants(layout):
    """insert_and_find_test.cpp:106-147: one winner per key and every
    duplicate returns the winner's payload."""
    import b2co
    import torch
    kb, vb = layout
    b, probing, hk = SCHEMES[0]
    rng = np.random.default_rng(99 + kb + vb)
    uniq = unique_keys(rng, 5000, kb)
    keys = rng.choice(uniq, size=60000)  # heavy duplication and contention
    vals = values_for(rng, keys, vb)
    t = make_table(kb, vb, b, probing, hk, 20000)
    found = out_buf(len(keys), kb, vb)
    inserted = torch.empty(len(keys), dtype=torch.uint8, device="cuda")
    t.InsertAndFind(make_pairs(keys, vals), found, inserted, mode=b2co.IAF_RACE)
    f, ins = found.cpu().numpy(), inserted.cpu().numpy()
    present = np.unique(keys)
    assert ins.sum() == len(present)
    for k in present[:500]:
        idx = np.nonzero(keys == k)[0]
        assert ins[idx].sum() == 1
        winner = idx[ins[idx] == 1][0]
        exp = keys[winner] if vb == 0 else vals[winner]
        assert (f[idx] == exp).all()


@pytest.mark.parametrize("layout", [l for l in LAYOUTS if l[1]], ids=lambda l: f"k{l[0]}v{l[1]}")
def test_insert_or_assign_and_assign_if_parity(layout):
    kb, vb = layout
    b, probing, hk = SCHEMES[0]
    rng = np.random.default_rng(515)
    keys = unique_keys(rng, 30000, kb)
    vals = values_for(rng, keys, vb)
    t = make_table(kb, vb, b, probing, hk, 60000)
    o = oracle_table(t, kb, vb, b, probing, hk)
    assert t.Insert(make_pairs(keys[:15000], vals[:15000])) == 0
    o.insert(keys[:15000], vals[:15000])
    upd = keys[10000:25000]
    uvals = values_for(rng, upd, vb)
    f, a = t.InsertOrAssign(make_pairs(upd, uvals), with_assigned=True)
    ef, ea = o.insert_or_assign(upd, uvals)
    assert (f, a) == (ef, ea) == (0, 5000)
    got, _ = stored_pairs(t, kb, vb, b, probing, hk)
    assert np.array_equal(got, o.pairs())
    # AssignIf: only selected existing keys change; absent keys are not inserted
    ak = np.concatenate([keys[:2000], keys[28000:]])
    av = values_for(rng, ak, vb)
    st = (rng.random(len(ak)) < 0.5).astype(np.uint8)
    t.AssignIfAsync(make_pairs(ak, av), dev(st))
    o.assign_if(ak, av, st)
    got, _ = stored_pairs(t, kb, vb, b, probing, hk)
    assert np.array_equal(got, o.pairs())


@pytest.mark.parametrize("layout", LAYOUTS, ids=lambda l: f"k{l[0]}v{l[1]}")
@pytest.mark.parametrize("tombstone", [False, True])
def test_erase_parity(layout, tombstone):
    kb, vb = layout
    b, probing, hk = SCHEMES[1] if not tombstone else SCHEMES[0]
    rng = np.random.default_rng(31 + kb + vb)
    keys = unique_keys(rng, 8000, kb)
    vals = values_for(rng, keys, vb)
    erased = -2 if tombstone else None
    t = make_table(kb, vb, b, probing, hk, 12000, erased_key=erased)
    o = oracle_table(t, kb, vb, b, probing, hk, erased_key=erased)
    t.Insert(make_pairs(keys, vals))
    o.insert(keys, vals)
    got, _ = stored_pairs(t, kb, vb, b, probing, hk, erased_key=erased)
    assert np.array_equal(got, o.pairs())
    # Later lookups depend on where erased slots sit in probe sequences, so
    # erase from identical slot positions: the oracle takes the device layout.
    o.load_slots(t.dump_slots())
    gone = np.concatenate([keys[:3000], miss_keys(rng, 500, kb)])
    assert t.Erase(dev(gone)) == o.erase(gone) == 500
    q = np.concatenate([keys, gone])
    out = out_buf(len(q), kb, vb)
    t.Find(dev(q), out)
    exp, _ = o.find(q)
    assert np.array_equal(out.cpu().numpy(), exp)
    got, _ = stored_pairs(t, kb, vb, b, probing, hk, erased_key=erased)
    assert np.array_equal(got, o.pairs())


@pytest.mark.parametrize("layout", [(4, 4), (8, 8), (8, 0)], ids=lambda l: f"k{l[0]}v{l[1]}")
def test_full_table(layout):
    """A full table rejects the overflow; every stored key is still found."""
    kb, vb = layout
    b, probing, hk = SCHEMES[0]
    rng = np.random.default_rng(8)
    t = make_table(kb, vb, b, probing, hk, 100)
    cap = t.Capacity()
    keys = unique_keys(rng, cap + 77, kb)
    vals = values_for(rng, keys, vb)
    assert t.Insert(make_pairs(keys, vals)) == 77
    import torch
    c = torch.empty(len(keys), dtype=torch.uint8, device="cuda")
    t.Contains(dev(keys), c)
    assert int(c.sum()) == cap
    assert t.Count(dev(miss_keys(rng, 50, kb))) == 0


@pytest.mark.parametrize("layout", [(4, 4), (8, 8), (8, 0)], ids=lambda l: f"k{l[0]}v{l[1]}")
def test_staged_shapes_on_full_table(layout):
    """Staged lookups of a full table: a miss follows every window of its probe
    cycle (the deferred shape queues it again window after window until the
    cycle closes), hits settle anywhere along the way.  Checked against the
    oracle reading the device table's own slots."""
    import torch
    kb, vb = layout
    b, probing, hk = SCHEMES[0]
    rng = np.random.default_rng(21)
    t = make_table(kb, vb, b, probing, hk, 300)
    keys = unique_keys(rng, t.Capacity() + 40, kb)
    t.Insert(make_pairs(keys, values_for(rng, keys, vb)))
    _, o = stored_pairs(t, kb, vb, b, probing, hk)
    q = np.concatenate([keys, miss_keys(rng, 3000, kb)])
    rng.shuffle(q)
    qd = dev(q)
    ref = (o.find(q)[0], o.contains(q)[0])
    for shape in [(2, 2, False, False, False, True), (4, 4, False, False, False, True),
                  (8, 1, False, False, False, True), (2, 2, False, False, True, False), (2, 2, False, False, False, False)]:
        t.set_find_shape(*shape)
        out = out_buf(len(q), kb, vb)
        t.Find(qd, out)
        c = torch.empty(len(q), dtype=torch.uint8, device="cuda")
        t.Contains(qd, c)
        assert np.array_equal(out.cpu().numpy(), ref[0]), shape
        assert np.array_equal(c.cpu().numpy(), ref[1]), shape


def test_edge_cases_and_errors():
    import b2co
    import torch
    t = b2co.StaticMap(1000, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64, probing=b2co.PROBE_DOUBLE,
                       hash_kind=b2co.HASH_XXH32)
    empty = torch.empty((0, 2), dtype=torch.int64, device="cuda")
    assert t.Insert(empty) == 0
    assert t.Insert(None, n=5) == 5          # NULL input: all items failed (open_addressing_impl.h:178-180)
    t.InsertAsync(None, n=5)                 # async: no-op
    p = b2co.pack_pairs(torch.tensor([-1, 7], device="cuda"), torch.tensor([3, 4], device="cuda"))
    assert t.Insert(p) == 1                  # the empty key is never inserted
    f = torch.empty(2, dtype=torch.int64, device="cuda")
    i = torch.empty(2, dtype=torch.uint8, device="cuda")
    t.InsertAndFind(p, f, i)
    assert f.tolist() == [-1, 4] and i.tolist() == [0, 0]
    with pytest.raises(b2co.LengthError):
        t.FindAsync(torch.zeros(1, dtype=torch.int64, device="cuda"), f, n=1 << 32)
    with pytest.raises(b2co.InvalidArgument):
        t.set_find_shape(3, 1)


def test_find_shapes_agree():
    import b2co
    import torch
    rng = np.random.default_rng(3)
    for kb, vb, b in [(8, 8, 5), (4, 4, 5), (8, 0, 8), (4, 8, 2)]:
        t = make_table(kb, vb, b, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, 300000)
        keys = unique_keys(rng, 200000, kb)   # high load: many second windows
        vals = values_for(rng, keys, vb)
        t.Insert(make_pairs(keys, vals))
        q = np.concatenate([keys[::3], miss_keys(rng, 50000, kb)])
        qd = dev(q)
        o = oracle_table(t, kb, vb, b, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
        o.insert(keys, vals)
        ref = (o.find(q)[0], o.contains(q)[0])
        shapes = [(l, i, False, False, False, False) for l in (1, 2, 4, 8) for i in (1, 2, 4)] + \
                 [(l, i, True, False, False, False) for l in (2, 4, 8) for i in (1, 2, 4)] + \
                 [(l, i, False, False, True, False) for l in (2, 4, 8) for i in (1, 2, 4)] + \
                 [(l, i, False, False, False, True) for l in (2, 4, 8) for i in (1, 2, 4)] + \
                 [(1, 1, False, True, False, False)]
        for lanes, items, seg, bulk, warp, defer in shapes:
            t.set_find_shape(lanes, items, seg, bulk, warp, defer)
            out = out_buf(len(q), kb, vb)
            t.Find(qd, out)
            c = torch.empty(len(q), dtype=torch.uint8, device="cuda")
            t.Contains(qd, c)
            assert np.array_equal(out.cpu().numpy(), ref[0]), (kb, vb, b, lanes, items, seg)
            assert np.array_equal(c.cpu().numpy(), ref[1]), (kb, vb, b, lanes, items, seg)


def test_find_host_buffers_match_device_find():
    import torch
    rng = np.random.default_rng(12)
    t = make_table(8, 8, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, 1 << 20)
    keys = unique_keys(rng, 1 << 19, 8)
    vals = values_for(rng, keys, 8)
    t.Insert(make_pairs(keys, vals))
    q = np.concatenate([keys, miss_keys(rng, 1 << 19, 8)])
    rng.shuffle(q)
    pinned_q = torch.from_numpy(q).pin_memory()
    pinned_o = torch.empty(len(q), dtype=torch.int64).pin_memory()
    t.FindHost(pinned_q.numpy(), pinned_o.numpy())
    out = out_buf(len(q), 8, 8)
    t.Find(dev(q), out)
    assert np.array_equal(pinned_o.numpy(), out.cpu().numpy())
    # a batch of 16 Mi keys or more ramps its chunk sizes up and down (1, 2, 4, ..., 2, 1 Mi keys)
    big = q[rng.integers(0, len(q), size=(17 << 20) + 5)]
    pinned_q = torch.from_numpy(big).pin_memory()
    pinned_o = torch.empty(len(big), dtype=torch.int64).pin_memory()
    t.FindHost(pinned_q.numpy(), pinned_o.numpy())
    out = out_buf(len(big), 8, 8)
    t.Find(dev(big), out)
    assert np.array_equal(pinned_o.numpy(), out.cpu().numpy())


def test_window_gather_measurement_aid():
    """The bare window-read measurement runs over 16- and 8-byte-slot tables,
    leaves the table unchanged, keeps the batch bound and refuses other slots."""
    import b2co
    import torch
    rng = np.random.default_rng(4)
    t = make_table(8, 8, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, 1 << 16)
    keys = unique_keys(rng, 20000, 8)
    t.Insert(make_pairs(keys, keys))
    before = t.dump_slots()
    t.window_gather(1 << 20, seed=3)
    torch.cuda.synchronize()
    assert np.array_equal(t.dump_slots(), before)
    with pytest.raises(b2co.LengthError):
        t.window_gather((1 << 31) + 1)
    m = make_table(4, 4, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, 1 << 16)
    k4 = unique_keys(rng, 20000, 4).astype(np.int32)
    m.Insert(make_pairs(k4, k4))
    before = m.dump_slots()
    m.window_gather(1 << 20, seed=5)
    torch.cuda.synchronize()
    assert np.array_equal(m.dump_slots(), before)
    s = make_table(4, 0, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, 1 << 12)
    with pytest.raises(b2co.InvalidArgument):
        s.window_gather(1024)
