"""Pins the StaticMultiset / StaticMultimap oracle (oracle/multi.py) to the
known answers in the reference's own tests:
tests/static_multimap/contract_test.cpp:18-133 and
tests/static_multiset/semantics_test.cpp (exact order, short outputs, predicate
selection, reserved key).  Sentinels are numeric_limits<T>::lowest(), as in
tests/common/static_multimap_test_common.h:98-107."""
import numpy as np
import pytest

from oracle.multi import InvalidArgument, LengthError, Multimap, Multiset


@pytest.mark.parametrize("dt", [np.int32, np.int64])
def test_multimap_contract_order(dt):
    lo = int(np.iinfo(dt).min)
    pairs = [(3, 9), (-7, 4), (3, -8), (3, -8), (-7, -3), (9, 7), (3, 2)]
    queries = [3, -7, 3, 42, lo]
    for _ in range(3):
        pairs = pairs[1:] + pairs[:1]  # std::rotate by one, as the test does each round
        m = Multimap(7, lo, lo, dt, dt)
        assert m.insert([p[0] for p in pairs], [p[1] for p in pairs]) == 0
        assert m.find(queries).tolist() == [-8, -3, -8, lo, lo]
        assert m.count(queries) == 10
        k, v = m.retrieve(queries, 10)
        assert k.tolist() == [3, 3, 3, 3, -7, -7, 3, 3, 3, 3]
        assert v.tolist() == [-8, -8, 2, 9, -3, 4, -8, -8, 2, 9]
        ak, av = m.retrieve_all(7)
        assert list(zip(ak.tolist(), av.tolist())) == pairs


@pytest.mark.parametrize("dt", [np.int32, np.int64])
def test_multimap_validation_and_prefix(dt):
    lo = int(np.iinfo(dt).min)
    m = Multimap(8, lo, lo, dt, dt)
    keys, vals = [1, 2, lo], [4, lo, 7]
    with pytest.raises(InvalidArgument):
        m.insert(keys, vals)
    assert m.size() == 0
    assert m.insert(keys, vals, stencil=[1, 0, 0]) == 0
    assert m.size() == 1
    with pytest.raises(LengthError):
        m.retrieve([1, 1], 1)
    with pytest.raises(LengthError):
        m.retrieve_all(0)
    # selected prefix (contract_test.cpp:56-94): 66049 pairs, every third unselected, capacity 513
    n = 66049
    st = [int(i % 3 != 0) for i in range(n)]
    m = Multimap(513, lo, lo, dt, dt)
    assert m.insert([i + 1 for i in range(n)], [i + 7 for i in range(n)], st) == sum(st) - 513
    ak, _ = m.retrieve_all(513)
    assert ak.tolist() == [i + 1 for i in range(n) if st[i]][:513]
    m = Multimap(513, lo, lo, dt, dt)
    assert m.insert([i + 1 for i in range(n)], [i + 7 for i in range(n)]) == n - 513
    assert m.retrieve_all(513)[0].tolist() == list(range(1, 514))


@pytest.mark.parametrize("dt", [np.int32, np.int64])
def test_multiset_exact_order(dt):
    lo, hi = int(np.iinfo(dt).min), int(np.iinfo(dt).max)
    keys = [7, 2, 7, hi, -4, 2, 9]
    s = Multiset(5, lo, dt)
    assert s.insert(keys) == 2
    assert s.retrieve_all(8).tolist() == keys[:5]
    q = [7, 8, 7, -4]
    assert s.count(q) == 5
    p, mt = s.retrieve(q, 8)
    assert p.tolist() == [7, 7, 7, 7, -4] and mt.tolist() == p.tolist()
    with pytest.raises(LengthError):
        s.retrieve_all(4)
    with pytest.raises(LengthError):
        s.retrieve(q, 4)


@pytest.mark.parametrize("dt", [np.int32, np.int64])
def test_multiset_predicate_and_reserved_key(dt):
    lo = int(np.iinfo(dt).min)
    keys = [3, lo, 3, 8, 9, -2]
    cond = [3, 4, 5, 1, 0, 6]
    s = Multiset(8, lo, dt)
    assert s.insert(keys, stencil=[c >= 3 for c in cond]) == 1
    assert s.size() == 3
    assert s.count_each(keys).tolist() == [2, 0, 2, 0, 0, 1]
    assert s.find(keys, stencil=[c >= 5 for c in cond]).tolist() == [lo, lo, 3, lo, lo, -2]
    assert s.count_each(keys, outer=True).tolist() == [2, 1, 2, 1, 1, 1]
