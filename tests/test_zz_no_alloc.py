"""The allocation-free InsertAndFind entry point, called through the C ABI.

It serves callers that cannot let the library allocate device memory (an
application that owns all device memory through its own arena, or a
latency-critical path that must not pay for an allocation); it takes its
scratch from a fixed device array inside the library.  Its results must equal
those of the regular first-wins InsertAndFind (exact: integer outputs), on two
calls in a row, whether this file runs alone in a fresh process or after the
rest of the suite.  This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from helpers import dev, unique_keys

pytestmark = pytest.mark.gpu


def _table(capacity):
    import b2co
    import torch
    return b2co.StaticMap(capacity, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64, bucket_size=5,
                          probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)


def _batch(rng, fresh, pre, n_dups):
    dups = rng.choice(np.concatenate([fresh, pre]), size=n_dups)
    keys = np.concatenate([fresh, dups, np.array([-1], dtype=np.int64)])
    rng.shuffle(keys)
    vals = rng.integers(0, 2**62, size=len(keys), dtype=np.int64)
    return keys, vals


def test_noalloc_insert_and_find_equals_regular_entry_point():
    import b2co
    import torch
    L = b2co.lib()
    L.b2co_oa_insert_and_find_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                                  C.c_void_p]
    rng = np.random.default_rng(2718)
    keys_all = unique_keys(rng, 300000, 8)
    ref, noa = _table(600000), _table(600000)
    seen = np.empty(0, dtype=np.int64)
    for call, (lo, hi) in enumerate([(0, 150000), (150000, 300000)]):   # two calls in a row
        keys, vals = _batch(rng, keys_all[lo:hi], seen[:20000], 30000)
        pairs = b2co.pack_pairs(dev(keys), dev(vals))
        n = len(keys)
        f_ref = torch.empty(n, dtype=torch.int64, device="cuda")
        i_ref = torch.empty(n, dtype=torch.uint8, device="cuda")
        ref.InsertAndFind(pairs, f_ref, i_ref, mode=b2co.IAF_FIRST_WINS)
        f_noa = torch.full((n,), 7, dtype=torch.int64, device="cuda")
        i_noa = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
        st = L.b2co_oa_insert_and_find_noalloc(noa._h, C.c_void_p(pairs.data_ptr()), C.c_void_p(f_noa.data_ptr()),
                                               C.c_void_p(i_noa.data_ptr()), C.c_uint64(n),
                                               C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 0, L.b2co_last_error()
        assert torch.equal(f_noa, f_ref), f"call {call}: found payloads differ"
        assert torch.equal(i_noa, i_ref), f"call {call}: inserted flags differ"
        assert int(i_noa.sum()) == len(np.setdiff1d(np.unique(keys[keys != -1]), seen))
        seen = np.concatenate([seen, keys_all[lo:hi]])
    # both tables hold the same pair set
    from helpers import stored_pairs
    import oracle
    a, _ = stored_pairs(ref, 8, 8, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    b, _ = stored_pairs(noa, 8, 8, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32)
    assert np.array_equal(a, b)


def test_noalloc_rejects_batches_beyond_its_scratch():
    import b2co
    import torch
    L = b2co.lib()
    big = _table(20_000_000)  # 4 bytes of scratch per slot alone exceed the fixed area
    pairs = torch.zeros((16, 2), dtype=torch.int64, device="cuda")
    f = torch.empty(16, dtype=torch.int64, device="cuda")
    i = torch.empty(16, dtype=torch.uint8, device="cuda")
    st = L.b2co_oa_insert_and_find_noalloc(big._h, C.c_void_p(pairs.data_ptr()), C.c_void_p(f.data_ptr()),
                                           C.c_void_p(i.data_ptr()), C.c_uint64(16), None)
    assert st == b2co.ERANGE
    assert b"scratch" in L.b2co_last_error()
