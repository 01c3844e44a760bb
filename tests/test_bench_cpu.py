"""Host-side pieces of bench.py that need no GPU."""
import bench


def test_host_find_chunk_schedule():
    """The host-buffer Find's chunk schedule (mirrored from b2co_oa_find_host):
    chunks cover the batch exactly, none is larger than 4 Mi keys, and batches
    of 16 Mi keys or more start with 1 and 2 Mi and end with 2 and 1 Mi."""
    full = 1 << 22
    assert bench.host_find_chunks(1) == 1
    assert bench.host_find_chunks(full) == 1
    assert bench.host_find_chunks(full + 1) == 2
    assert bench.host_find_chunks(4 * full - 1) == 4
    # 2^27 keys: 1, 2, thirty of 4, 2, 2, 1 (Mi keys)
    assert bench.host_find_chunks(1 << 27) == 35
    for n in (4 * full, 4 * full + 5, (17 << 20) + 5, 1 << 27, (1 << 27) + 12345):
        count = bench.host_find_chunks(n)
        # at most two extra chunks at each end over the uniform schedule
        assert (n + full - 1) // full <= count <= (n + full - 1) // full + 4
