"""The benchmark workloads checked exactly at their stated sizes.

Every other GPU test compares the CUDA path with the oracle on inputs the
oracle finishes in well under a second.  This file runs the very inputs the
benchmark times -- generated by bench.py's own generators -- at full size and
compares every output with the oracle:

* StaticMap<int64,int64>, 2^28 requested slots (268,728,155), DoubleHashing
  <xxhash_32>, bucket 5, filled by first-wins InsertAndFind to load factor 0.5
  (149,293,419 inputs, 10% duplicates) and 0.8: found values and inserted
  flags against the oracle's sequential fill (the golden of
  tests/common/golden.h:104-131), the stored pair set against the oracle
  table, and Find/Contains on full 2^27-query streams at 0/50/100% hits and
  Zipf(1.1);
* BloomFilter: 2^22 blocks, 2^28 adds -- the whole 128 MiB word array and all
  2^28 Contains outputs (bloom_filter_test.cpp:205-230 compares the same);
* HyperLogLog<int64>, p = 16: 2^30 adds over 10^7 distinct keys as one sketch
  and as 16 sub-sketches merged -- registers identical to the oracle's
  (add_test.cpp:321-398), Estimate equal to the FP64 finalizer;
* 4,096 batched StaticMap<int32,int32> tables: every table's stored set and
  every Find output against the oracle rebuilding each table on its own.

The oracle's read-only checks run on all host threads.  Slow by design
(minutes); marked gpu like the other parity tests.
"""
import os
import sys

import numpy as np
import pytest

import oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
import bench  # noqa: E402  (the benchmark's own input generators)

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1


def _map88(capacity):
    import b2co
    import torch
    return b2co.StaticMap(capacity, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64, bucket_size=5,
                          probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)


@pytest.mark.parametrize("lf", [0.5, 0.8])
def test_cfg2_first_wins_fill_stored_set_and_queries_exact(lf):
    import b2co
    import torch
    t = _map88(1 << 28)
    cap = t.Capacity()
    assert cap == 268_728_155
    unique, dups = bench.workload_sizes(cap, lf)
    keys, stream, vals = bench.make_insert_stream(unique, dups, "torch")
    pairs = b2co.pack_pairs(stream, vals)
    found = torch.empty(stream.numel(), dtype=torch.int64, device="cuda")
    ins = torch.empty(stream.numel(), dtype=torch.uint8, device="cuda")
    t.InsertAndFind(pairs, found, ins, mode=b2co.IAF_FIRST_WINS)
    del pairs
    s_h, v_h = stream.cpu().numpy(), vals.cpu().numpy()
    del stream, vals

    o = oracle.Table(np.int64, np.int64, cap, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    exp_found, exp_ins = o.insert_and_find(s_h, v_h)
    del s_h, v_h
    assert int(exp_ins.sum()) == unique
    assert np.array_equal(ins.cpu().numpy(), exp_ins), "inserted flags differ from the sequential golden"
    assert np.array_equal(found.cpu().numpy(), exp_found), "found values differ from the sequential golden"
    del found, ins, exp_found, exp_ins

    d = oracle.Table(np.int64, np.int64, cap, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    d.load_slots(t.dump_slots())
    equal, n_o, n_d, mism = o.same_pairs(d, THREADS)
    assert equal, f"stored pair sets differ: oracle {n_o}, device {n_d}, {mism} oracle pairs missing or changed"
    assert n_o == unique
    del d

    n = 1 << 27
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    flags = torch.empty(n, dtype=torch.uint8, device="cuda")
    streams = [(0.5, None)] if lf != 0.5 else [(0.0, None), (0.5, None), (1.0, None), (1.0, 1.1)]
    for hr, zipf in streams:
        q = bench.make_queries(keys, n, hr, "torch", zipf_s=zipf)
        t.Find(q, out)
        t.Contains(q, flags)
        q_h = q.cpu().numpy()
        del q
        exp = o.find_parallel(q_h, THREADS)
        assert np.array_equal(out.cpu().numpy(), exp), f"Find differs (hits {hr}, zipf {zipf})"
        exp_c = o.contains_parallel(q_h, THREADS)
        assert np.array_equal(flags.cpu().numpy(), exp_c), f"Contains differs (hits {hr}, zipf {zipf})"
        if zipf is None:
            assert abs(float(exp_c.mean()) - hr) < 1e-3


def test_cfg3_bloom_word_array_and_all_queries_exact():
    import b2co
    import torch
    g = torch.Generator(device="cuda").manual_seed(bench.SEED + 7)
    nb, adds, q = bench.bloom_workload(g)
    f = b2co.BloomFilter(nb, key_dtype=torch.int64)
    f.Add(adds)
    out = torch.empty(q.numel(), dtype=torch.uint8, device="cuda")
    f.Contains(q, out)
    words = np.zeros(nb * 8, np.uint32)
    oracle.bloom_add(words, nb, adds.cpu().numpy())
    assert np.array_equal(f.words(), words), "Bloom word arrays differ"
    exp = oracle.bloom_contains(words, nb, q.cpu().numpy(), threads=THREADS)
    assert np.array_equal(out.cpu().numpy(), exp), "Bloom Contains outputs differ"
    assert exp[: q.numel() // 2].all()  # the first half are added keys


def test_cfg3_hll_registers_merge_and_estimate_exact():
    import b2co
    import torch
    g = torch.Generator(device="cuda").manual_seed(bench.SEED + 7)
    n, parts = 1 << 30, 16
    keys = bench.hll_keys(g, n)
    one = b2co.HyperLogLog(16)
    one.Add(keys)
    subs = [b2co.HyperLogLog(16) for _ in range(parts)]
    reg = np.zeros(1 << 16, np.uint8)
    step = n // parts
    for i, sub in enumerate(subs):
        sub.Add(keys[i * step:(i + 1) * step])
        oracle.hll_add(reg, 16, keys[i * step:(i + 1) * step].cpu().numpy(), threads=THREADS)
    del keys
    for sub in subs[1:]:
        subs[0].Merge(sub)
    assert np.array_equal(one.registers(), reg), "one-shot registers differ from the oracle"
    assert np.array_equal(subs[0].registers(), reg), "merged sub-sketch registers differ from the oracle"
    hist = oracle.hll_histogram(reg, 16)
    assert np.array_equal(one.Histogram(), hist)
    raw, bias, thr = b2co.hll_bias_data(16)
    exact = oracle.hll_finalize(16, hist, raw, bias, thr)
    assert one.Estimate() == exact and subs[0].Estimate() == exact
    assert abs(exact - 10_000_000) / 10_000_000 < 0.01


def test_cfg4_every_batched_table_exact():
    import b2co
    import torch
    w = bench.batched_workload()
    sizes, ins_off, q_off = w["sizes"], w["ins_off"], w["q_off"]
    grp = b2co.TableGroup(2 * sizes, -1, -1, key_dtype=torch.int32, value_dtype=torch.int32)
    assert grp.Insert(w["pairs"], torch.from_numpy(ins_off).cuda()) == 0
    out = torch.empty(w["queries"].numel(), dtype=torch.int32, device="cuda")
    grp.Find(w["queries"], torch.from_numpy(q_off).cuda(), out)
    caps = np.array([grp.table_capacity(t) for t in range(len(sizes))], dtype=np.uint64)
    assert all(int(c) == oracle.valid_capacity(int(2 * s), 5, oracle.PROBE_DOUBLE) for c, s in zip(caps, sizes))
    shape = oracle.Table(np.int32, np.int32, 5, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    bad, first, expected = oracle.group_check(caps, shape, grp.dump_slots(), w["keys"].cpu().numpy(),
                                              w["vals"].cpu().numpy(), ins_off, w["queries"].cpu().numpy(), q_off,
                                              THREADS)
    assert bad == 0, f"{bad} tables store another pair set than the oracle's (first: table {first})"
    assert np.array_equal(out.cpu().numpy(), expected), "batched Find outputs differ from the oracle"
    hit = w["hit"].cpu().numpy()
    assert np.array_equal(expected != -1, hit)
