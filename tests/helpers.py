"""Shared helpers for the GPU parity tests: seeded inputs and conversion
between the product's device tables and the oracle's host tables."""
import numpy as np

import oracle

NP_DT = {4: np.int32, 8: np.int64}
LAYOUTS = [(4, 0), (8, 0), (4, 4), (4, 8), (8, 4), (8, 8)]


def torch_dt(nbytes):
    import torch
    return {4: torch.int32, 8: torch.int64}[nbytes]


def unique_keys(rng, n, kb, lo=0, hi=None):
    """n distinct keys, never the -1 sentinel (generators.h style: uniform draws).
    The default range [0, 2^30) (4-byte) / [0, 2^62) (8-byte) never meets miss_keys()."""
    hi = hi if hi is not None else (2**30 if kb == 4 else 2**62)
    out = np.unique(rng.integers(lo, hi, size=int(n * 1.3) + 16, dtype=np.int64))
    rng.shuffle(out)
    out = out[:n]
    assert len(out) == n
    return out.astype(NP_DT[kb])


def miss_keys(rng, n, kb):
    """n distinct keys from a range disjoint from unique_keys()' default range."""
    return unique_keys(rng, n, kb, lo=2**30 if kb == 4 else 2**62, hi=2**31 - 2 if kb == 4 else 2**63 - 2)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def make_pairs(keys_np, vals_np):
    """Device Pair<K,V> array for a map, or the key array for a set."""
    import b2co
    k = dev(keys_np)
    if vals_np is None:
        return k
    return b2co.pack_pairs(k, dev(vals_np))


def oracle_table(gpu_table, kb, vb, bucket_size, probing, hash_kind, empty_key=-1, empty_value=-1, erased_key=None):
    return oracle.Table(NP_DT[kb], None if vb == 0 else NP_DT[vb], gpu_table.Capacity(), bucket_size, probing,
                        hash_kind, empty_key, empty_value, erased_key)


def stored_pairs(gpu_table, kb, vb, bucket_size, probing, hash_kind, erased_key=None):
    """The device table's stored pair set, read through an oracle table of the same layout."""
    t = oracle_table(gpu_table, kb, vb, bucket_size, probing, hash_kind, erased_key=erased_key)
    t.load_slots(gpu_table.dump_slots())
    return t.pairs(), t
