"""Failure detection without a GPU fault: the staged lookup kernels wait on
their own bulk key copies with a time limit.  The test hook makes the first
wait of every block be on a barrier that nothing ever arrives on; the kernel
must give up after the limit, record the timeout, let its copies land and
return, the call must report ETIMEOUT, and the context must stay usable."""
import ctypes as C

import numpy as np
import pytest

from helpers import dev, unique_keys

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(8, 4, False, False, False), (1, 1, False, True, False),
                                   (2, 2, False, False, True), (2, 2, False, False, False, True)],
                         ids=["staged", "bulk", "warp_staged", "deferred"])
def test_bounded_wait_reports_timeout_and_context_survives(shape):
    import b2co
    import torch
    rng = np.random.default_rng(17)
    t = b2co.StaticMap(100000, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64, probing=b2co.PROBE_DOUBLE,
                       hash_kind=b2co.HASH_XXH32)
    t.set_find_shape(*shape)  # the staged / bulk-window kernels wait on their own bulk copies
    keys = unique_keys(rng, 50000, 8)
    t.Insert(b2co.pack_pairs(dev(keys), dev(keys)))
    q = dev(keys[:8192])
    out = torch.empty(8192, dtype=torch.int64, device="cuda")
    L = b2co.lib()
    try:
        assert L.b2co_debug_set_wait(C.c_uint64(5_000_000), 1) == 0   # 5 ms limit, wait on a dead barrier
        with pytest.raises(b2co.TimeoutError_):
            t.Find(q, out)
    finally:
        L.b2co_debug_set_wait(C.c_uint64(0), 0)
    # the status word was cleared by the report; the next lookup is correct
    t.Find(q, out)
    assert np.array_equal(out.cpu().numpy(), keys[:8192])
    torch.cuda.synchronize()
