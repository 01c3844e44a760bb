"""Table groups (the batched pattern): many StaticMap<int32,int32> tables of
uneven sizes, inserted and queried by one persistent launch, by its CUDA-graph
replay and by one plain launch per table -- all identical to the oracle run
table by table."""
import numpy as np
import pytest

import oracle
from helpers import dev

pytestmark = pytest.mark.gpu


def build_workload(rng, count):
    sizes = np.clip(np.exp2(rng.normal(np.log2(3000), 1.5, size=count)), 64, 40000).astype(np.int64)
    keys, vals, queries = [], [], []
    for n in sizes:
        k = rng.choice(np.arange(0, 2**30, dtype=np.int64), size=n, replace=False) if n > 5000 else \
            np.unique(rng.integers(0, 2**30, size=int(n * 1.2) + 8))[:n]
        rng.shuffle(k)
        k = k[:n].astype(np.int32)
        keys.append(k)
        vals.append(rng.integers(0, 2**31 - 2, size=len(k)).astype(np.int32))
        miss = rng.integers(2**30, 2**31 - 2, size=len(k)).astype(np.int32)
        q = np.concatenate([rng.choice(k, size=len(k)), miss])
        rng.shuffle(q)
        queries.append(q)
    sizes = np.array([len(k) for k in keys])
    ins_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    q_off = np.concatenate([[0], np.cumsum([len(q) for q in queries])]).astype(np.uint64)
    return sizes, keys, vals, queries, ins_off, q_off


def test_group_insert_find_graph_per_table_match_oracle(tmp_path):
    import b2co
    import torch
    rng = np.random.default_rng(404)
    count = 60
    sizes, keys, vals, queries, ins_off, q_off = build_workload(rng, count)
    caps = 2 * sizes
    g = b2co.TableGroup(caps, -1, -1, key_dtype=torch.int32, value_dtype=torch.int32)
    pairs = b2co.pack_pairs(dev(np.concatenate(keys)), dev(np.concatenate(vals)))
    assert g.Insert(pairs, dev(ins_off.astype(np.int64))) == 0

    slab = g.dump_slots()
    qcat = np.concatenate(queries)
    expected = []
    off = 0
    for t in range(count):
        cap = g.table_capacity(t)
        assert cap == oracle.valid_capacity(int(caps[t]), 5, oracle.PROBE_DOUBLE)
        o = oracle.Table(np.int32, np.int32, cap, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
        assert o.insert(keys[t], vals[t]) == 0
        dev_t = oracle.Table(np.int32, np.int32, cap, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
        dev_t.load_slots(slab[off * 8:(off + cap) * 8])
        assert np.array_equal(dev_t.pairs(), o.pairs()), t
        expected.append(o.find(queries[t])[0])
        off += cap
    expected = np.concatenate(expected)

    qd = dev(qcat)
    d_qoff = dev(q_off.astype(np.int64))
    shapes = [(1, 1, 0), (2, 1, 0), (4, 1, 0), (8, 1, 0), (2, 2, 256), (4, 2, 0), (4, 4, 128), (8, 2, 256),
              (8, 4, 64)]
    for shape in shapes:  # every shape, deferred or not, block sizes included
        g.set_find_shape(*shape)
        out = torch.empty(len(qcat), dtype=torch.int32, device="cuda")
        g.Find(qd, d_qoff, out)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), expected), shape
        c = torch.empty(len(qcat), dtype=torch.uint8, device="cuda")
        g.Find(qd, d_qoff, c, contains=True)
        assert np.array_equal(c.cpu().numpy(), (expected != -1).astype(np.uint8)), shape
    out = torch.empty(len(qcat), dtype=torch.int32, device="cuda")
    g.Find(qd, d_qoff, out, graph=True)
    g.Find(qd, d_qoff, out, graph=True)  # replay
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), expected)
    out = torch.empty(len(qcat), dtype=torch.int32, device="cuda")
    g.FindPerTable(qd, q_off, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), expected)
    c = torch.empty(len(qcat), dtype=torch.uint8, device="cuda")
    g.Find(qd, d_qoff, c, contains=True)
    torch.cuda.synchronize()
    assert np.array_equal(c.cpu().numpy(), (expected != -1).astype(np.uint8))
    b2co.tune_cache_clear()
    out = torch.empty(len(qcat), dtype=torch.int32, device="cuda")
    shape, cached = g.Autotune(qd, d_qoff, out)
    assert not cached and shape[0] in (1, 2, 4, 8) and shape == g.find_shape()
    assert np.array_equal(out.cpu().numpy(), expected)
    # the choice is reused without timing, and survives a save / clear / load round trip
    out = torch.empty(len(qcat), dtype=torch.int32, device="cuda")
    assert g.Autotune(qd, d_qoff, out) == (shape, True)
    assert np.array_equal(out.cpu().numpy(), expected)
    path = str(tmp_path / "tune.txt")
    b2co.tune_cache_save(path)
    b2co.tune_cache_clear()
    b2co.tune_cache_load(path)
    g.set_find_shape(1)
    assert g.Autotune(qd, d_qoff, out) == (shape, True) and g.find_shape() == shape

    # the per-table insert path builds the same tables
    g2 = b2co.TableGroup(caps, -1, -1, key_dtype=torch.int32, value_dtype=torch.int32)
    g2.InsertPerTable(pairs, ins_off)
    torch.cuda.synchronize()
    out = torch.empty(len(qcat), dtype=torch.int32, device="cuda")
    g2.Find(qd, d_qoff, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), expected)
