"""CPU oracle for StaticMultiset / StaticMultimap (numpy restatement).

TEST INFRASTRUCTURE ONLY, like the rest of ``oracle/``: the checker for the
CUDA containers in ``ops-collections_b200``, never part of the product.

These containers expose no slot layout (no ``Data()``), so their results are
defined by the multiset of stored entries and the reference's ordering rules,
which this module restates:

* StaticMultiset<Key> (include/static_multiset.h):
  - Insert / InsertIf (:159-190, :473-534): among the selected keys, the empty
    key is a failure; the earliest valid keys up to the remaining capacity are
    kept, in input order; failed = valid - accepted + sentinel keys.  A null
    key array with n > 0 returns n and changes nothing.
  - Contains / Find / CountEach / CountEachOuter (:192-260): per-key
    multiplicity; Find writes the key or the empty key; Outer replaces 0 by 1;
    the If forms write 0 / the empty key for unselected inputs.
  - Count (:290-294): sum of multiplicities over all query positions.
  - Retrieve (:296-321): for each query in order, `count` copies of
    (query, query); a too-small output is a length error and writes nothing.
  - RetrieveAll (:322-343): every stored key in accepted insertion order.
* StaticMultimap<Key, Value> (include/static_multimap.h):
  - Insert / InsertIf (:288-399, :430-460): every selected pair is validated
    first (a sentinel key or value -> invalid_argument, nothing inserted);
    then the earliest selected pairs up to the remaining capacity are kept;
    duplicates (even identical pairs) are retained; failed = selected - accepted.
  - Find (static_multimap_ref.h QueryImpl): the smallest value stored under the
    key, else the empty value (also for the empty key).
  - Contains / Count: existence / total matches over all query positions.
  - Retrieve (:493-510): per query in order, its values in ascending order.
  - RetrieveAll (:512-553): all pairs; the dense storage keeps accepted
    insertion order (contract_test.cpp:194-240), which this oracle returns.
"""
from __future__ import annotations

from collections import Counter, defaultdict

import numpy as np


class LengthError(Exception):
    pass


class InvalidArgument(Exception):
    pass


class Multiset:
    def __init__(self, capacity: int, empty_key: int, dtype=np.int64):
        self.capacity, self.empty, self.dtype = capacity, int(empty_key), np.dtype(dtype)
        self.ordered: list[int] = []
        self.counts: Counter = Counter()

    def insert(self, keys, stencil=None) -> int:
        keys = [int(k) for k in keys]
        sel = [True] * len(keys) if stencil is None else [bool(s) for s in stencil]
        valid = [k for k, s in zip(keys, sel) if s and k != self.empty]
        invalid = sum(1 for k, s in zip(keys, sel) if s and k == self.empty)
        accepted = min(len(valid), self.capacity - len(self.ordered))
        for k in valid[:accepted]:
            self.ordered.append(k)
            self.counts[k] += 1
        return len(valid) - accepted + invalid

    def size(self) -> int:
        return len(self.ordered)

    def count_each(self, keys, outer=False):
        out = np.array([0 if int(k) == self.empty else self.counts.get(int(k), 0) for k in keys], dtype=np.uint64)
        return np.maximum(out, 1) if outer else out

    def contains(self, keys, stencil=None):
        c = self.count_each(keys)
        s = np.ones(len(c), bool) if stencil is None else np.asarray(stencil).astype(bool)
        return ((c > 0) & s).astype(np.uint8)

    def find(self, keys, stencil=None):
        c = self.count_each(keys)
        s = np.ones(len(c), bool) if stencil is None else np.asarray(stencil).astype(bool)
        k = np.asarray(keys, dtype=self.dtype)
        return np.where((c > 0) & s, k, np.array(self.empty, dtype=self.dtype)).astype(self.dtype)

    def count(self, keys) -> int:
        return int(self.count_each(keys).sum())

    def retrieve(self, keys, out_capacity: int):
        c = self.count_each(keys)
        total = int(c.sum())
        if total > out_capacity:
            raise LengthError(total)
        probe = np.repeat(np.asarray(keys, dtype=self.dtype), c.astype(np.int64))
        return probe, probe.copy()

    def retrieve_all(self, out_capacity: int):
        if len(self.ordered) > out_capacity:
            raise LengthError(len(self.ordered))
        return np.array(self.ordered, dtype=self.dtype)


class Multimap:
    def __init__(self, capacity: int, empty_key: int, empty_value: int, key_dtype=np.int64, value_dtype=np.int64):
        self.capacity, self.ek, self.ev = capacity, int(empty_key), int(empty_value)
        self.kdt, self.vdt = np.dtype(key_dtype), np.dtype(value_dtype)
        self.pairs: list[tuple[int, int]] = []
        self.values = defaultdict(list)

    def insert(self, keys, values, stencil=None) -> int:
        keys, values = [int(k) for k in keys], [int(v) for v in values]
        sel = [True] * len(keys) if stencil is None else [bool(s) for s in stencil]
        chosen = [(k, v) for k, v, s in zip(keys, values, sel) if s]
        if any(k == self.ek or v == self.ev for k, v in chosen):
            raise InvalidArgument("a selected pair holds a reserved key or value")
        accepted = min(len(chosen), self.capacity - len(self.pairs))
        for k, v in chosen[:accepted]:
            self.pairs.append((k, v))
            self.values[k].append(v)
        return len(chosen) - accepted

    def size(self) -> int:
        return len(self.pairs)

    def _vals(self, k):
        k = int(k)
        return [] if k == self.ek else sorted(self.values.get(k, []))

    def contains(self, keys, stencil=None):
        s = np.ones(len(keys), bool) if stencil is None else np.asarray(stencil).astype(bool)
        return np.array([bool(self._vals(k)) and bool(si) for k, si in zip(keys, s)], dtype=np.uint8)

    def find(self, keys, stencil=None):
        s = np.ones(len(keys), bool) if stencil is None else np.asarray(stencil).astype(bool)
        out = [(self._vals(k)[0] if self._vals(k) else self.ev) if si else self.ev for k, si in zip(keys, s)]
        return np.array(out, dtype=self.vdt)

    def count(self, keys) -> int:
        return sum(len(self._vals(k)) for k in keys)

    def retrieve(self, keys, out_capacity: int):
        total = self.count(keys)
        if total > out_capacity:
            raise LengthError(total)
        pk, pv = [], []
        for k in keys:
            vs = self._vals(k)
            pk += [int(k)] * len(vs)
            pv += vs
        return np.array(pk, dtype=self.kdt), np.array(pv, dtype=self.vdt)

    def retrieve_all(self, out_capacity: int):
        if len(self.pairs) > out_capacity:
            raise LengthError(len(self.pairs))
        return (np.array([p[0] for p in self.pairs], dtype=self.kdt),
                np.array([p[1] for p in self.pairs], dtype=self.vdt))
