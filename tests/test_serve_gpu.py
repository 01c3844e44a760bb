"""The request server (served pattern): requests of uneven sizes against two
resident StaticMap<int64,int64> tables, Finds and InsertOrAssigns mixed.

Each request's result must be the same when it runs alone (one request at a
time) as when it runs in the mix (many in flight, Finds coalesced), and equal
to the oracle replaying the requests in arrival order: a Find sees exactly the
InsertOrAssigns that arrived before it on its table (upserted keys are queried
by later Finds and re-assigned by later upserts).  Admission by the HBM budget:
a request that can never fit is rejected, a tight budget serializes."""
import numpy as np
import pytest

import oracle
from helpers import dev, unique_keys

pytestmark = pytest.mark.gpu

N_TABLES = 2
N_INITIAL = 600_000


def initial_contents():
    rng = np.random.default_rng(11)
    out = []
    for _ in range(N_TABLES):
        keys = unique_keys(rng, N_INITIAL, 8).astype(np.int64)
        vals = rng.integers(0, 2**62, size=N_INITIAL)
        out.append((keys, vals))
    return out


def make_requests(contents, count=64, seed=5):
    """(table, op, payload): 1 in 6 an InsertOrAssign of fresh keys plus some
    keys earlier upserts wrote; Finds of log-normal sizes hit initial keys,
    upserted keys, and keys no request ever writes."""
    import b2co
    rng = np.random.default_rng(seed)
    reqs = []
    upserted = [np.zeros(0, np.int64) for _ in range(N_TABLES)]
    fresh = 2**62 + 1000  # upsert keys: [2^62, 2^62 + 2^40); misses: [2^62 + 2^61, 2^63)
    for i in range(count):
        t = int(rng.integers(0, N_TABLES))
        if i % 6 == 5:
            n_new = int(rng.integers(1000, 20000))
            k = np.arange(fresh, fresh + n_new, dtype=np.int64)
            fresh += n_new
            if len(upserted[t]):
                again = rng.choice(upserted[t], size=min(len(upserted[t]), 3000), replace=False)
                k = np.concatenate([k, again])
            rng.shuffle(k)
            v = rng.integers(0, 2**62, size=len(k))
            reqs.append((t, b2co.OP_INSERT_OR_ASSIGN, np.stack([k, v], axis=1).astype(np.int64)))
            upserted[t] = np.unique(np.concatenate([upserted[t], k]))
        else:
            n = int(np.clip(np.exp(rng.normal(np.log(8000), 1.2)), 1000, 200000))
            keys, _ = contents[t]
            pick = rng.random(n)
            q = keys[rng.integers(0, len(keys), size=n)]
            if len(upserted[t]):
                q = np.where(pick < 0.2, upserted[t][rng.integers(0, len(upserted[t]), size=n)], q)
            miss = rng.integers(2**62 + 2**61, 2**63 - 2, size=n)
            q = np.where(pick > 0.7, miss, q).astype(np.int64)
            reqs.append((t, b2co.OP_FIND, q))
    return reqs


def expected(contents, reqs, capacity):
    """The oracle replaying every request in arrival order."""
    import b2co
    tabs = []
    for keys, vals in contents:
        o = oracle.Table(np.int64, np.int64, capacity, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
        assert o.insert(keys, vals) == 0
        tabs.append(o)
    outs, counts = [], []
    for t, op, data in reqs:
        if op == b2co.OP_FIND:
            outs.append(tabs[t].find(data)[0])
            counts.append(None)
        else:
            outs.append(None)
            counts.append(tabs[t].insert_or_assign(data[:, 0], data[:, 1]))
    return outs, counts, [o.pairs() for o in tabs]


def make_tables(contents):
    import b2co
    import torch
    tables = []
    for keys, vals in contents:
        m = b2co.StaticMap(1_000_000, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64,
                           probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)
        assert m.Insert(b2co.pack_pairs(dev(keys), dev(vals))) == 0
        tables.append(m)
    torch.cuda.synchronize()
    return tables


def run(contents, reqs, max_inflight, sequential, max_batch_keys=0, packing=False, plain=False, direct=True):
    """Runs the requests through a server; `direct` (results written by the
    GPU into the pinned result buffers) is on here so the default test covers
    that path, the other modes are switched explicitly."""
    import b2co
    tables = make_tables(contents)
    srv = b2co.Server(max_inflight=max_inflight, hbm_budget_bytes=8 << 30, max_batch_keys=max_batch_keys)
    srv.set_packing(packing)
    srv.set_plain(plain)
    srv.set_direct_results(direct)
    for m in tables:
        srv.register(m)
    ins, bufs, infos, ids = [], [], [], []
    for t, op, data in reqs:
        inp = b2co.pinned(data.shape, np.int64)
        inp[...] = data
        ins.append(inp)
        bufs.append(b2co.pinned((len(data),), np.int64) if op == b2co.OP_FIND else None)
    # the mix: every request arrives at one instant shortly after submission
    at = 0 if sequential else b2co.Server.now_ns() + 20_000_000
    for (t, op, _), inp, out in zip(reqs, ins, bufs):
        rid = srv.submit(tables[t], op, inp, out, arrival_ns=at)
        if sequential:
            infos.append(srv.wait(rid))
        else:
            ids.append(rid)
    infos += [srv.wait(rid) for rid in ids]
    stats = srv.stats()
    srv.close()
    outs = [None if b is None else b.copy() for b in bufs]
    pairs = []
    for m in tables:
        o = oracle.Table(np.int64, np.int64, m.Capacity(), 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
        o.load_slots(m.dump_slots())
        pairs.append(o.pairs())
    return outs, infos, pairs, stats, tables[0].Capacity()


def test_results_same_alone_and_in_the_mix():
    import b2co
    contents = initial_contents()
    reqs = make_requests(contents)
    a_out, a_info, a_pairs, a_stats, cap = run(contents, reqs, 1, sequential=True)
    b_out, b_info, b_pairs, b_stats, _ = run(contents, reqs, 8, sequential=False)
    e_out, e_counts, e_pairs = expected(contents, reqs, cap)
    for i, (t, op, data) in enumerate(reqs):
        if op == b2co.OP_FIND:
            assert np.array_equal(a_out[i], e_out[i]), i
            assert np.array_equal(b_out[i], e_out[i]), i
        else:
            assert (a_info[i].failed, a_info[i].assigned) == e_counts[i], i
            assert (b_info[i].failed, b_info[i].assigned) == e_counts[i], i
    for x, y, e in zip(a_pairs, b_pairs, e_pairs):
        assert np.array_equal(x, e) and np.array_equal(y, e)
    assert all(i.status == 0 for i in a_info + b_info)
    assert all(i.done_ns >= i.admit_ns >= i.arrival_ns for i in b_info)
    assert sum(c[1] for c in e_counts if c) > 0  # some upserts re-assigned earlier upserts
    # one launch per request alone; the mix coalesced Finds
    assert a_stats["launches"] == len(reqs)
    assert b_stats["launches"] < len(reqs)
    assert b_stats["requests_launched"] == len(reqs)
    # staging was sized at creation: no buffer grew under traffic
    assert b_stats["staging_grows"] == 8
    # lookups took their results straight from the GPU: no copy out, so fewer copies than two per request
    assert b_stats["direct_launches"] > 0 and a_stats["direct_launches"] > 0
    assert b_stats["copies"] < 2 * len(reqs)


def test_mix_copied_packed_and_plain_modes_give_the_same_results():
    """The coalescing server with results copied out per request, with
    coalesced requests packed into one copy each way, and the plain baseline
    (one launch per request, one request per table at a time; results copied
    out or written directly) give the sequential results too."""
    import b2co
    contents = initial_contents()
    reqs = make_requests(contents)
    e_out = None
    for kw in ({"direct": False}, {"direct": False, "packing": True}, {"plain": True, "direct": False},
               {"plain": True}):
        out, info, pairs, stats, cap = run(contents, reqs, 8, sequential=False, **kw)
        if e_out is None:
            e_out, e_counts, e_pairs = expected(contents, reqs, cap)
        for i, (t, op, data) in enumerate(reqs):
            if op == b2co.OP_FIND:
                assert np.array_equal(out[i], e_out[i]), (kw, i)
            else:
                assert (info[i].failed, info[i].assigned) == e_counts[i], (kw, i)
        for x, e in zip(pairs, e_pairs):
            assert np.array_equal(x, e), kw
        assert (stats["packed_launches"] > 0) == bool(kw.get("packing")), kw
        assert (stats["direct_launches"] > 0) == kw.get("direct", True), kw
        if kw.get("plain"):
            assert stats["launches"] == len(reqs)


def test_scheduled_arrivals_and_small_batches():
    """Arrival times in the future (a Poisson schedule) submitted in two
    batched calls, and a max batch below most request sizes: results
    unchanged, latency measured from arrival."""
    import b2co
    contents = initial_contents()
    reqs = make_requests(contents, count=24, seed=9)
    e_out, _, _ = expected(contents, reqs, b2co.valid_capacity(1_000_000))
    tables = make_tables(contents)
    srv = b2co.Server(max_inflight=4, hbm_budget_bytes=8 << 30, max_batch_keys=4096)
    for m in tables:
        srv.register(m)
    rng = np.random.default_rng(3)
    t0 = b2co.Server.now_ns() + 20_000_000
    arrivals = t0 + np.cumsum(rng.exponential(200_000, size=len(reqs))).astype(np.int64)
    ins, bufs = [], []
    descs = np.zeros(len(reqs), dtype=b2co.REQUEST_DESC)
    for i, ((t, op, data), at) in enumerate(zip(reqs, arrivals)):
        inp = b2co.pinned(data.shape, np.int64)
        inp[...] = data
        out = b2co.pinned((len(data),), np.int64) if op == b2co.OP_FIND else None
        ins.append(inp)
        bufs.append(out)
        descs[i] = (tables[t]._h.value, op, 0, inp.ctypes.data, 0 if out is None else out.ctypes.data, len(data), at)
    ids = np.concatenate([srv.submit_many(descs[:10]), srv.submit_many(descs[10:])])
    infos = srv.wait_many(ids)
    srv.close()
    assert (infos["id"] == ids).all() and (infos["status"] == 0).all()
    for i, (info, at) in enumerate(zip(infos, arrivals)):
        assert info["arrival_ns"] == at and info["admit_ns"] >= at and info["done_ns"] >= info["admit_ns"]
        if e_out[i] is not None:
            assert np.array_equal(bufs[i], e_out[i]), i
    with pytest.raises(b2co.InvalidArgument):  # arrival order is the submission order
        srv2 = b2co.Server(max_inflight=1, hbm_budget_bytes=8 << 30)
        srv2.register(tables[0])
        q = b2co.pinned((1000,), np.int64)
        o = b2co.pinned((1000,), np.int64)
        now = b2co.Server.now_ns()
        srv2.submit(tables[0], b2co.OP_FIND, q, o, arrival_ns=now + 10_000_000)
        try:
            srv2.submit(tables[0], b2co.OP_FIND, q, o, arrival_ns=now + 5_000_000)
        finally:
            srv2.close()


def test_waits_in_any_order_while_requests_stay_queued():
    """Plain mode admits requests out of queue order, so a finished request can
    stay in the dispatcher's queue after its caller waited for it.  Here the
    caller waits newest first and submits more in between (new requests may
    reuse freed memory); every result stays right in both modes, because a
    request is freed only when the queue and the caller have both let it go."""
    import b2co
    contents = initial_contents()
    reqs = [r for r in make_requests(contents, count=120, seed=21) if r[1] == b2co.OP_FIND]
    e_out, _, _ = expected(contents, reqs, b2co.valid_capacity(1_000_000))
    tables = make_tables(contents)
    half = len(reqs) // 2
    for plain in (True, False):
        srv = b2co.Server(max_inflight=4, hbm_budget_bytes=8 << 30)
        srv.set_plain(plain)
        for m in tables:
            srv.register(m)
        ins, outs, ids = [], [], []
        at = b2co.Server.now_ns() + 10_000_000

        def submit(i):
            t, op, data = reqs[i]
            inp = b2co.pinned(data.shape, np.int64)
            inp[...] = data
            out = b2co.pinned((len(data),), np.int64)
            ins.append(inp)
            outs.append(out)
            ids.append(srv.submit(tables[t], op, inp, out, arrival_ns=at))

        for i in range(half):
            submit(i)
        for k in range(half):
            srv.wait(ids[half - 1 - k])
            submit(half + k)
        for rid in ids[half:]:
            srv.wait(rid)
        srv.close()
        for i in range(len(reqs)):
            assert np.array_equal(outs[i], e_out[i]), (plain, i)


def test_budget_admission():
    import b2co
    import torch
    m = b2co.StaticMap(100000, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64)
    table_bytes = m.Capacity() * 16 + 24
    with pytest.raises(b2co.BadAlloc):
        b2co.Server(hbm_budget_bytes=table_bytes - 1).register(m)
    # room for the table plus about three 20k-key lookups at a time
    srv = b2co.Server(max_inflight=4, hbm_budget_bytes=table_bytes + (1 << 20))
    srv.register(m)
    big = b2co.pinned((200000,), np.int64)
    big[:] = np.arange(200000)
    out_big = b2co.pinned((200000,), np.int64)
    rid = srv.submit(m, b2co.OP_FIND, big, out_big)
    with pytest.raises(b2co.BadAlloc):
        srv.wait(rid)  # 3.2 MB of staging can never fit a 1 MiB budget
    small = [b2co.pinned((20000,), np.int64) for _ in range(6)]
    outs = [b2co.pinned((20000,), np.int64) for _ in range(6)]
    for s in small:
        s[:] = np.arange(20000)
    ids = [srv.submit(m, b2co.OP_FIND, s, o) for s, o in zip(small, outs)]
    infos = [srv.wait(i) for i in ids]
    assert all(i.status == 0 for i in infos)
    assert all((o == -1).all() for o in outs)
    # resident table plus the staging buffers the slots kept, never above the budget
    assert table_bytes < srv.stats()["bytes_in_use"] <= table_bytes + (1 << 20)
    srv.close()
