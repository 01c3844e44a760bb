"""GPU parity tests for BloomFilter and HyperLogLog through the C ABI against
the oracle: identical bit arrays and per-query results
(tests/bloom_filter/bloom_filter_test.cpp:205-230), identical HLL registers
(tests/hyperloglog/add_test.cpp:321-398) and Estimate equal to the FP64 host
finalizer."""
import numpy as np
import pytest

import oracle
from helpers import dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["atomic", "bulk", "partitioned", "auto"])
@pytest.mark.parametrize("kdt", [np.uint32, np.int32, np.uint64, np.int64, np.float32])
@pytest.mark.parametrize("num_blocks", [1, 7, 4096, 5000, 1 << 16])
def test_bloom_add_contains_bit_exact(kdt, num_blocks, mode):
    """Every Add path of the default policy (64-bit atomics, TMA bulk ORs, keys
    routed by filter slice, and the automatic choice) sets exactly the oracle's
    bits; 4096 blocks is one whole slice, 5000 ends in a partial one."""
    import b2co
    import torch
    rng = np.random.default_rng(int(num_blocks) + np.dtype(kdt).itemsize)
    n = 50000
    if np.dtype(kdt).kind == "f":
        keys = rng.standard_normal(n).astype(kdt)
        keys[:4] = [0.0, -0.0, np.inf, -np.inf]   # signed zeros hash their bit patterns
    else:
        keys = rng.integers(0, np.iinfo(kdt).max, size=n, dtype=np.uint64).astype(kdt)
    ktorch = {np.uint32: torch.int32, np.int32: torch.int32, np.float32: torch.int32,
              np.uint64: torch.int64, np.int64: torch.int64}[kdt]
    f = b2co.BloomFilter(num_blocks, key_dtype=ktorch)
    f.set_add_mode({"atomic": b2co.BLOOM_ADD_ATOMIC, "bulk": b2co.BLOOM_ADD_BULK,
                    "partitioned": b2co.BLOOM_ADD_PARTITIONED, "auto": b2co.BLOOM_ADD_AUTO}[mode])
    kd = torch.from_numpy(keys.view(np.int32 if keys.itemsize == 4 else np.int64)).cuda()
    f.Add(kd[: n // 2])
    f.AddAsync(kd[n // 2:])
    words = np.zeros(num_blocks * 8, dtype=np.uint32)
    oracle.bloom_add(words, num_blocks, keys)
    assert np.array_equal(f.words(), words)
    q = np.concatenate([keys[::5], rng.integers(0, 2**31, size=20000).astype(kdt)])
    qd = torch.from_numpy(q.view(np.int32 if q.itemsize == 4 else np.int64)).cuda()
    out = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    f.Contains(qd, out)
    assert np.array_equal(out.cpu().numpy(), oracle.bloom_contains(words, num_blocks, q))
    assert out[: len(keys[::5])].all()  # no false negatives
    st = (rng.random(len(q)) < 0.5).astype(np.uint8)
    f.ContainsIf(qd, dev(st), out)
    assert np.array_equal(out.cpu().numpy(), oracle.bloom_contains(words, num_blocks, q) & st)


def test_partitioned_adds_on_two_streams_share_the_workspace_in_order():
    """Two asynchronous routed Adds on different streams use the filter's one
    workspace one after the other; the bits are the oracle's for both batches."""
    import b2co
    import torch
    rng = np.random.default_rng(31)
    nb = 5000
    ka = rng.integers(0, 2**63, size=400000, dtype=np.uint64)
    kb = rng.integers(0, 2**63, size=300000, dtype=np.uint64)
    f = b2co.BloomFilter(nb, key_dtype=torch.int64)
    f.set_add_mode(b2co.BLOOM_ADD_PARTITIONED)
    da, db = dev(ka.view(np.int64)), dev(kb.view(np.int64))
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    f.AddAsync(da, stream=s1)
    f.AddAsync(db, stream=s2)
    torch.cuda.synchronize()
    words = np.zeros(nb * 8, dtype=np.uint32)
    oracle.bloom_add(words, nb, ka)
    oracle.bloom_add(words, nb, kb)
    assert np.array_equal(f.words(), words)
    # AddIf on the routed path: only selected keys set bits
    kc = rng.integers(0, 2**63, size=200000, dtype=np.uint64)
    st = (rng.random(len(kc)) < 0.3).astype(np.uint8)
    f.AddIf(dev(kc.view(np.int64)), dev(st))
    oracle.bloom_add(words, nb, kc[st.astype(bool)])
    assert np.array_equal(f.words(), words)


def test_bloom_add_if_merge_intersect_and_errors():
    import b2co
    import torch
    rng = np.random.default_rng(2)
    nb = 1024
    a, b = b2co.BloomFilter(nb), b2co.BloomFilter(nb)
    ka = rng.integers(0, 2**63, size=30000, dtype=np.uint64)
    kb = rng.integers(0, 2**63, size=30000, dtype=np.uint64)
    st = (rng.random(len(ka)) < 0.4).astype(np.uint8)
    a.AddIf(dev(ka.view(np.int64)), dev(st))
    b.Add(dev(kb.view(np.int64)))
    wa = np.zeros(nb * 8, np.uint32)
    oracle.bloom_add(wa, nb, ka[st.astype(bool)])
    wb = np.zeros(nb * 8, np.uint32)
    oracle.bloom_add(wb, nb, kb)
    assert np.array_equal(a.words(), wa)
    a.Merge(b)
    assert np.array_equal(a.words(), wa | wb)
    a.Intersect(b)
    assert np.array_equal(a.words(), (wa | wb) & wb)
    with pytest.raises(b2co.InvalidArgument):
        a.Merge(b2co.BloomFilter(nb + 1))
    with pytest.raises(b2co.InvalidArgument):
        a.Merge(b2co.BloomFilter(nb, seed=3))
    with pytest.raises(b2co.InvalidArgument):
        a.Add(None, n=10)
    a.Add(None, n=0)  # zero keys: no-op
    a.Clear()
    assert not a.words().any()


POLICIES = [(1, 1), (1, 32), (2, 2), (2, 64), (4, 4), (4, 16), (8, 16), (8, 64), (16, 16), (16, 48), (32, 32),
            (32, 64)]


@pytest.mark.parametrize("policy", POLICIES, ids=lambda p: f"w{p[0]}p{p[1]}")
@pytest.mark.parametrize("key_bytes", [4, 8])
def test_bloom_policy_bit_exact(policy, key_bytes):
    """Non-default BloomFilterPolicy (WordsPerBlock, PatternBits), as in the
    reference's generalization_test.cpp: the bit array after Add and AddIf, the
    results of Contains and ContainsIf, Merge and Intersect all equal the oracle."""
    import b2co
    import torch
    wpb, pbits = policy
    rng = np.random.default_rng(wpb * 100 + pbits + key_bytes)
    kdt = np.uint32 if key_bytes == 4 else np.uint64
    tdt = torch.int32 if key_bytes == 4 else torch.int64
    vdt = np.int32 if key_bytes == 4 else np.int64
    for nb, seed in [(257, 42), (1 << 16, 0)]:
        n = 40000
        keys = rng.integers(0, np.iinfo(kdt).max, size=n, dtype=np.uint64).astype(kdt)
        keys[n // 2:n // 2 + 1000] = keys[:1000]  # repeated keys
        f = b2co.BloomFilter(nb, key_dtype=tdt, seed=seed, words_per_block=wpb, pattern_bits=pbits)
        st = (rng.random(n) < 0.6).astype(np.uint8)
        f.Add(dev(keys[: n // 2].view(vdt)))
        f.AddIf(dev(keys[n // 2:].view(vdt)), dev(st[n // 2:]))
        words = np.zeros(nb * wpb, dtype=np.uint32)
        oracle.bloom_add(words, nb, keys[: n // 2], seed, wpb, pbits)
        oracle.bloom_add(words, nb, keys[n // 2:][st[n // 2:].astype(bool)], seed, wpb, pbits)
        assert np.array_equal(f.words(), words)
        q = np.concatenate([keys[::7], rng.integers(0, np.iinfo(kdt).max, size=20000, dtype=np.uint64).astype(kdt)])
        out = torch.empty(len(q), dtype=torch.uint8, device="cuda")
        f.Contains(dev(q.view(vdt)), out)
        exp = oracle.bloom_contains(words, nb, q, seed, 1, wpb, pbits)
        assert np.array_equal(out.cpu().numpy(), exp)
        qs = (rng.random(len(q)) < 0.5).astype(np.uint8)
        f.ContainsIf(dev(q.view(vdt)), dev(qs), out)
        assert np.array_equal(out.cpu().numpy(), exp & qs)
        g = b2co.BloomFilter(nb, key_dtype=tdt, seed=seed, words_per_block=wpb, pattern_bits=pbits)
        other = keys[: n // 3][::-1].copy()
        g.Add(dev(other.view(vdt)))
        wg = np.zeros_like(words)
        oracle.bloom_add(wg, nb, other, seed, wpb, pbits)
        f.Merge(g)
        assert np.array_equal(f.words(), words | wg)
        f.Intersect(g)
        assert np.array_equal(f.words(), (words | wg) & wg)
        with pytest.raises(b2co.InvalidArgument):  # same blocks, different policy
            f.Merge(b2co.BloomFilter(nb, key_dtype=tdt, seed=seed, words_per_block=wpb * 2 if wpb < 32 else 16,
                                     pattern_bits=64))
        f.Clear()
        assert not f.words().any()


def test_bloom_policy_arguments():
    import b2co
    import torch
    for wpb, pbits in [(3, 3), (64, 64), (8, 4), (8, 12), (4, 80), (1, 33), (0, 8)]:
        with pytest.raises(b2co.InvalidArgument):
            b2co.BloomFilter(16, key_dtype=torch.int64, words_per_block=wpb, pattern_bits=pbits)
    # the default filter and an explicit (8, 8) filter (ArrowFilterPolicy) are the same filter
    keys = np.arange(1, 5001, dtype=np.int64) * 2654435761
    a = b2co.BloomFilter(333, key_dtype=torch.int64)
    b = b2co.BloomFilter(333, key_dtype=torch.int64, words_per_block=8, pattern_bits=8)
    a.Add(dev(keys))
    b.Add(dev(keys))
    assert np.array_equal(a.words(), b.words())
    a.Merge(b)


@pytest.mark.parametrize("precision", [13, 14, 15, 16, 17, 18])
@pytest.mark.parametrize("key_bytes", [4, 8])
def test_hll_registers_bit_exact(precision, key_bytes):
    import b2co
    import torch
    rng = np.random.default_rng(precision * 10 + key_bytes)
    kdt = np.int32 if key_bytes == 4 else np.int64
    distinct = rng.integers(np.iinfo(kdt).min, np.iinfo(kdt).max, size=200000, dtype=np.int64).astype(kdt)
    keys = rng.choice(distinct, size=700000)
    h = b2co.HyperLogLog(precision, key_dtype=torch.int32 if key_bytes == 4 else torch.int64)
    kd = dev(keys)
    h.Add(kd[:100])          # tiny batch
    h.Add(kd[100:300001])    # medium, ragged end
    h.Add(kd[300001:])       # large, starts off a 16-byte boundary
    reg = np.zeros(1 << precision, np.uint8)
    oracle.hll_add(reg, precision, keys)
    assert np.array_equal(h.registers(), reg)
    hist = oracle.hll_histogram(reg, precision)
    assert np.array_equal(h.Histogram(), hist)
    raw, bias, thr = b2co.hll_bias_data(precision)
    est = h.Estimate()
    assert est == oracle.hll_finalize(precision, hist, raw, bias, thr)
    # accuracy band used by tests/common/hll_test_common.h:90-99
    true = len(np.unique(keys))
    assert abs(est - true) <= 3 * 1.04 / np.sqrt(1 << precision) * true


def test_hll_merge_batched_equals_one_shot_and_errors():
    import b2co
    import torch
    rng = np.random.default_rng(9)
    keys = rng.integers(-2**62, 2**62, size=400000, dtype=np.int64)
    one = b2co.HyperLogLog.CreateWithSketchSizeKB(64)
    one.Add(dev(keys))
    parts = [b2co.HyperLogLog(16) for _ in range(4)]
    for i, p in enumerate(parts):
        p.Add(dev(keys[i::4]))
    for p in parts[1:]:
        parts[0].Merge(p)
    assert np.array_equal(parts[0].registers(), one.registers())
    assert parts[0].Estimate() == one.Estimate()
    with pytest.raises(b2co.InvalidArgument):
        parts[0].Merge(b2co.HyperLogLog(15))
    e = b2co.HyperLogLog(14)
    assert e.Estimate() == 0  # all registers zero: linear counting gives 0
    e.Add(None, n=0)
