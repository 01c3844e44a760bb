"""GPU parity tests for StaticMultiset / StaticMultimap through the C ABI
against the oracle (oracle/multi.py): the reference's contract cases
(tests/static_multimap/contract_test.cpp, tests/static_multiset/semantics_test.cpp)
and randomized workloads with heavy duplicate groups, stencils, capacity
overflow and every key / value width.  Outputs are compared exactly."""
import numpy as np
import pytest

from helpers import dev
from oracle.multi import InvalidArgument as OInvalid, LengthError as OLength, Multimap, Multiset

pytestmark = pytest.mark.gpu

TORCH = {4: "int32", 8: "int64"}
NP = {4: np.int32, 8: np.int64}


def tdt(nbytes):
    import torch
    return getattr(torch, TORCH[nbytes])


def pairs_dev(keys, values):
    import b2co
    return b2co.pack_pairs(dev(keys), dev(values))


def empty_dev(n, nbytes):
    import torch
    return torch.empty(max(n, 1), dtype=tdt(nbytes), device="cuda")


@pytest.mark.parametrize("kb,vb", [(4, 4), (4, 8), (8, 4), (8, 8)])
def test_multimap_contract_case(kb, vb):
    import b2co
    lo_k, lo_v = int(np.iinfo(NP[kb]).min), int(np.iinfo(NP[vb]).min)
    pairs = [(3, 9), (-7, 4), (3, -8), (3, -8), (-7, -3), (9, 7), (3, 2)]
    queries = np.array([3, -7, 3, 42, lo_k], dtype=NP[kb])
    m = b2co.StaticMultimap(7, lo_k, lo_v, key_dtype=tdt(kb), value_dtype=tdt(vb))
    for _ in range(3):
        pairs = pairs[1:] + pairs[:1]
        m.Clear()
        k = np.array([p[0] for p in pairs], NP[kb])
        v = np.array([p[1] for p in pairs], NP[vb])
        assert m.Insert(pairs_dev(k, v)) == 0
        found = empty_dev(5, vb)
        m.Find(dev(queries), found)
        assert found.cpu().numpy().tolist() == [-8, -3, -8, lo_v, lo_v]
        assert m.Count(dev(queries)) == 10
        ok, ov = empty_dev(10, kb), empty_dev(10, vb)
        assert m.Retrieve(dev(queries), ok, ov, 10) == 10
        assert ok.cpu().numpy().tolist() == [3, 3, 3, 3, -7, -7, 3, 3, 3, 3]
        assert ov.cpu().numpy().tolist() == [-8, -8, 2, 9, -3, 4, -8, -8, 2, 9]
        ak, av = empty_dev(7, kb), empty_dev(7, vb)
        assert m.RetrieveAll(ak, av, 7) == 7
        assert list(zip(ak.cpu().tolist(), av.cpu().tolist())) == pairs
    # validation preserves state and outputs
    m = b2co.StaticMultimap(8, lo_k, lo_v, key_dtype=tdt(kb), value_dtype=tdt(vb))
    bad = pairs_dev(np.array([1, 2, lo_k], NP[kb]), np.array([4, lo_v, 7], NP[vb]))
    with pytest.raises(b2co.InvalidArgument):
        m.Insert(bad)
    assert m.Size() == 0
    assert m.InsertIf(bad, dev(np.array([1, 0, 0], np.uint8))) == 0
    assert m.Size() == 1
    q = dev(np.array([1, 1], NP[kb]))
    ok, ov = empty_dev(2, kb), empty_dev(2, vb)
    ok.fill_(123)
    ov.fill_(123)
    with pytest.raises(b2co.LengthError):
        m.Retrieve(q, ok, ov, 1)
    assert ok.cpu().tolist() == [123, 123] and ov.cpu().tolist() == [123, 123]
    with pytest.raises(b2co.LengthError):
        m.RetrieveAll(ok, ov, 0)
    with pytest.raises(b2co.InvalidArgument):
        m.Find(None, ov, n=1)
    with pytest.raises(b2co.OverflowError_):
        m.Count(q, n=1 << 63)
    assert m.Size() == 1


@pytest.mark.parametrize("kb", [4, 8])
def test_multimap_selected_prefix(kb):
    import b2co
    lo = int(np.iinfo(NP[kb]).min)
    n = 66049
    st = np.array([i % 3 != 0 for i in range(n)], np.uint8)
    keys = np.arange(1, n + 1, dtype=NP[kb])
    vals = np.arange(7, n + 7, dtype=NP[kb])
    m = b2co.StaticMultimap(513, lo, lo, key_dtype=tdt(kb), value_dtype=tdt(kb))
    assert m.InsertIf(pairs_dev(keys, vals), dev(st)) == int(st.sum()) - 513
    ak, av = empty_dev(513, kb), empty_dev(513, kb)
    assert m.RetrieveAll(ak, av, 513) == 513
    assert ak.cpu().numpy().tolist() == keys[st.astype(bool)][:513].tolist()
    m.Clear()
    assert m.Insert(pairs_dev(keys, vals)) == n - 513
    m.RetrieveAll(ak, av, 513)
    assert ak.cpu().numpy().tolist() == list(range(1, 514))


@pytest.mark.parametrize("kb,vb", [(4, 4), (4, 8), (8, 4), (8, 8)])
def test_multimap_random_against_oracle(kb, vb):
    import b2co
    rng = np.random.default_rng(kb * 10 + vb)
    lo_k, lo_v = int(np.iinfo(NP[kb]).min), int(np.iinfo(NP[vb]).min)
    cap = 150_000
    m = b2co.StaticMultimap(cap, lo_k, lo_v, key_dtype=tdt(kb), value_dtype=tdt(vb))
    o = Multimap(cap, lo_k, lo_v, NP[kb], NP[vb])
    distinct = rng.integers(-2**30, 2**30, size=20000).astype(NP[kb])
    for batch in range(3):
        n = 70_000
        # skewed: a few keys with thousands of values, most with a handful
        idx = np.where(rng.random(n) < 0.1, rng.integers(0, 5, size=n), rng.integers(0, len(distinct), size=n))
        k = distinct[idx]
        v = rng.integers(-2**30, 2**30, size=n).astype(NP[vb])
        st = (rng.random(n) < 0.8).astype(np.uint8) if batch == 1 else None
        got = m.InsertIf(pairs_dev(k, v), dev(st)) if st is not None else m.Insert(pairs_dev(k, v))
        assert got == o.insert(k, v, st)
        assert m.Size() == o.size()
        q = np.concatenate([distinct[rng.integers(0, len(distinct), size=30000)],
                            rng.integers(-2**30, 2**30, size=5000).astype(NP[kb]), distinct[:5],
                            np.array([lo_k], NP[kb])])
        out = empty_dev(len(q), vb)
        m.Find(dev(q), out)
        assert np.array_equal(out.cpu().numpy(), o.find(q))
        c = dev(np.zeros(len(q), np.uint8))
        m.Contains(dev(q), c)
        assert np.array_equal(c.cpu().numpy(), o.contains(q))
        qs = (rng.random(len(q)) < 0.5).astype(np.uint8)
        m.FindIf(dev(q), dev(qs), out)
        assert np.array_equal(out.cpu().numpy(), o.find(q, qs))
        total = o.count(q)
        assert m.Count(dev(q)) == total
        qr = q[:2000]
        tr = o.count(qr)
        ok, ov = empty_dev(tr, kb), empty_dev(tr, vb)
        assert m.Retrieve(dev(qr), ok, ov, tr) == tr
        ek, ev = o.retrieve(qr, tr)
        assert np.array_equal(ok.cpu().numpy()[:tr], ek) and np.array_equal(ov.cpu().numpy()[:tr], ev)
    ak, av = empty_dev(cap, kb), empty_dev(cap, vb)
    assert m.RetrieveAll(ak, av, cap) == o.size()
    ek, ev = o.retrieve_all(cap)
    assert np.array_equal(ak.cpu().numpy()[:o.size()], ek) and np.array_equal(av.cpu().numpy()[:o.size()], ev)


@pytest.mark.parametrize("kb", [4, 8])
def test_multiset_contract_cases(kb):
    import b2co
    import torch
    lo, hi = int(np.iinfo(NP[kb]).min), int(np.iinfo(NP[kb]).max)
    keys = np.array([7, 2, 7, hi, -4, 2, 9], NP[kb])
    s = b2co.StaticMultiset(5, lo, key_dtype=tdt(kb))
    for _ in range(3):
        s.Clear()
        assert s.Insert(dev(keys)) == 2
        out = empty_dev(8, kb)
        assert s.RetrieveAll(out, 8) == 5
        assert out.cpu().numpy()[:5].tolist() == keys[:5].tolist()
        q = dev(np.array([7, 8, 7, -4], NP[kb]))
        assert s.Count(q) == 5
        pr, mt = empty_dev(8, kb), empty_dev(8, kb)
        assert s.Retrieve(q, pr, mt, 8) == 5
        assert pr.cpu().numpy()[:5].tolist() == [7, 7, 7, 7, -4] and mt.cpu().numpy()[:5].tolist() == [7, 7, 7, 7, -4]
        out.fill_(42)
        with pytest.raises(b2co.LengthError):
            s.RetrieveAll(out, 4)
        assert (out.cpu().numpy() == 42).all()
    keys = np.array([3, lo, 3, 8, 9, -2], NP[kb])
    cond = np.array([3, 4, 5, 1, 0, 6])
    s = b2co.StaticMultiset(8, lo, key_dtype=tdt(kb))
    assert s.InsertIf(dev(keys), dev((cond >= 3).astype(np.uint8))) == 1
    assert s.Size() == 3
    counts = torch.empty(6, dtype=torch.int64, device="cuda")
    s.CountEach(dev(keys), counts)
    assert counts.cpu().tolist() == [2, 0, 2, 0, 0, 1]
    found = empty_dev(6, kb)
    s.FindIf(dev(keys), dev((cond >= 5).astype(np.uint8)), found)
    assert found.cpu().tolist() == [lo, lo, 3, lo, lo, -2]
    s.CountEachOuter(dev(keys), counts)
    assert counts.cpu().tolist() == [2, 1, 2, 1, 1, 1]
    assert s.Insert(None, n=5) == 5  # a null key array: every key failed, nothing changes
    assert s.Size() == 3
    with pytest.raises(b2co.InvalidArgument):
        b2co.StaticMultiset(0, lo, key_dtype=tdt(kb))


@pytest.mark.parametrize("kb", [4, 8])
def test_multiset_random_against_oracle(kb):
    import b2co
    import torch
    rng = np.random.default_rng(77 + kb)
    lo = int(np.iinfo(NP[kb]).min)
    cap = 120_000
    s = b2co.StaticMultiset(cap, lo, key_dtype=tdt(kb))
    o = Multiset(cap, lo, NP[kb])
    distinct = rng.integers(-2**30, 2**30, size=10000).astype(NP[kb])
    for batch in range(3):
        n = 50_000
        k = distinct[np.where(rng.random(n) < 0.2, rng.integers(0, 3, size=n), rng.integers(0, len(distinct), size=n))]
        k[rng.random(n) < 0.01] = lo  # sentinel keys are failures
        st = (rng.random(n) < 0.7).astype(np.uint8) if batch == 2 else None
        got = s.InsertIf(dev(k), dev(st)) if st is not None else s.Insert(dev(k))
        assert got == o.insert(k, st)
        assert s.Size() == o.size()
    q = np.concatenate([distinct[rng.integers(0, len(distinct), size=20000)],
                        rng.integers(-2**30, 2**30, size=3000).astype(NP[kb]), np.array([lo], NP[kb])])
    counts = torch.empty(len(q), dtype=torch.int64, device="cuda")
    s.CountEach(dev(q), counts)
    assert np.array_equal(counts.cpu().numpy().astype(np.uint64), o.count_each(q))
    s.CountEachOuter(dev(q), counts)
    assert np.array_equal(counts.cpu().numpy().astype(np.uint64), o.count_each(q, outer=True))
    c = dev(np.zeros(len(q), np.uint8))
    s.Contains(dev(q), c)
    assert np.array_equal(c.cpu().numpy(), o.contains(q))
    f = empty_dev(len(q), kb)
    s.Find(dev(q), f)
    assert np.array_equal(f.cpu().numpy(), o.find(q))
    assert s.Count(dev(q)) == o.count(q)
    qr = q[:3000]
    tr = o.count(qr)
    pr, mt = empty_dev(tr, kb), empty_dev(tr, kb)
    assert s.Retrieve(dev(qr), pr, mt, tr) == tr
    ep, em = o.retrieve(qr, tr)
    assert np.array_equal(pr.cpu().numpy()[:tr], ep) and np.array_equal(mt.cpu().numpy()[:tr], em)
    out = empty_dev(cap, kb)
    assert s.RetrieveAll(out, cap) == o.size()
    assert np.array_equal(out.cpu().numpy()[:o.size()], o.retrieve_all(cap))
