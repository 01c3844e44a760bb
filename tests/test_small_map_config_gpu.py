"""The reference's own CPU-runnable workload at full size, bit-exact against
the oracle: StaticMap<int32,int32> with DoubleHashing<xxhash_32> and sentinels
-1, requested capacity 2,097,152 slots; 1,000,000 unique keys drawn uniformly
from [0, 2^31 - 2] (seed 1) with value = 2*key + 1; Find and Contains on
1,000,000 queries, half of them inserted keys and half from a disjoint range.
Both bucket sizes the reference's tests use (5 and 1)."""
import numpy as np
import pytest

import oracle
from helpers import dev, stored_pairs

pytestmark = pytest.mark.gpu

N = 1_000_000
REQUEST = 2_097_152


def workload():
    rng = np.random.default_rng(1)
    keys = np.unique(rng.integers(0, 2**31 - 1, size=int(N * 1.1), dtype=np.int64))
    rng.shuffle(keys)
    keys = keys[:N]
    assert len(keys) == N
    vals = ((2 * keys + 1) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)  # int32 wrap
    ins = set(keys.tolist())
    miss = rng.integers(0, 2**31 - 1, size=int(N * 0.6), dtype=np.int64)
    miss = np.unique(np.array([m for m in miss.tolist() if m not in ins], dtype=np.int64))[: N // 2]
    hits = keys[rng.integers(0, N, size=N // 2)]
    q = np.concatenate([hits, miss])
    rng.shuffle(q)
    return keys.astype(np.int32), vals, q.astype(np.int32)


@pytest.mark.parametrize("bucket,expected_capacity", [(5, 2_621_735), (1, 2_097_349)])
def test_small_map_workload_bit_exact(bucket, expected_capacity):
    import b2co
    import torch
    keys, vals, q = workload()
    m = b2co.StaticMap(REQUEST, -1, -1, key_dtype=torch.int32, value_dtype=torch.int32, bucket_size=bucket,
                       probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)
    assert m.Capacity() == expected_capacity
    o = oracle.Table(np.int32, np.int32, m.Capacity(), bucket, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    assert m.Insert(b2co.pack_pairs(dev(keys), dev(vals))) == 0
    assert o.insert(keys, vals) == 0
    dq = dev(q)
    out = torch.empty(len(q), dtype=torch.int32, device="cuda")
    m.Find(dq, out)
    flags = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    m.Contains(dq, flags)
    exp_out, _ = o.find(q)
    exp_flags, _ = o.contains(q)
    assert np.array_equal(out.cpu().numpy(), exp_out)
    assert np.array_equal(flags.cpu().numpy(), exp_flags)
    assert int(exp_flags.sum()) == N // 2
    got, _ = stored_pairs(m, 4, 4, bucket, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    assert np.array_equal(got, o.pairs())
