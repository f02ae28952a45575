"""The allocation-free compaction entry point (wrk_compact_noalloc).

Some callers cannot let a library allocate device memory -- a process that
reserved a fixed device-memory budget at start-up, or a framework whose allocator
must own every device byte.  wrk_compact_noalloc serves them with scratch built
into the library.  This file runs last (pytest collects it after the others), so
a failure here leaves every other result already reported; it also passes when
run alone in a fresh process.

Checked through the C ABI: the output equals wrk_compact's (the allocating entry
point) exactly -- compaction is integer work -- on two calls in a row, whose
inputs differ so the second call runs on the scratch the first one left behind.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _compact_via(entry, L, stage, idx):
    from offlinerenderer_b200 import wrk

    ds = wrk.DeviceArray.from_numpy(stage)
    di = wrk.DeviceArray.from_numpy(idx)
    do = wrk.DeviceArray((max(1, len(idx)),), np.uint32)
    dc = wrk.DeviceArray((1,), np.uint32)
    rc = getattr(L, entry)(ds.ptr, di.ptr, len(idx), do.ptr, dc.ptr)
    assert rc == 0, L.wrk_last_error()
    return do.numpy()[: int(dc.numpy()[0])]


def test_noalloc_compaction_matches_allocating_entry_point(gpu):
    L = gpu.lib()
    rng = np.random.default_rng(2024)
    # first call: a large ragged input; second call: a smaller one, so stale tile
    # counts from the first call sit in the shared scratch beyond the second's tiles
    for n in (3_000_001, 70_000):
        stage = rng.integers(0, 4, n).astype(np.uint32)
        idx = rng.permutation(n).astype(np.uint32)
        want = _compact_via("wrk_compact", L, stage, idx)
        got = _compact_via("wrk_compact_noalloc", L, stage, idx)
        assert np.array_equal(got, want), n
        assert np.array_equal(got, idx[stage[idx] != 3])


def test_noalloc_compaction_at_tile_boundaries(gpu):
    """Exact multiples of the 1024-entry tile: one tile, 1024 tiles (the scan's
    first carry into a second chunk of tile counts) and 65,536 tiles, the largest
    input the fixed scratch accepts (256 MiB per index buffer)."""
    L = gpu.lib()
    rng = np.random.default_rng(7)
    for n in (1024, 1024 * 1024, 1024 * 1024 + 1, 65536 * 1024):
        stage = rng.integers(0, 4, n, dtype=np.uint32)
        idx = rng.permutation(n).astype(np.uint32)
        got = _compact_via("wrk_compact_noalloc", L, stage, idx)
        assert np.array_equal(got, idx[stage[idx] != 3]), n
        want = _compact_via("wrk_compact", L, stage, idx)
        assert np.array_equal(got, want), n


def test_noalloc_compaction_rejects_sizes_beyond_its_scratch(gpu):
    L = gpu.lib()
    wrk = gpu
    small = wrk.DeviceArray((16,), np.uint32)
    count = wrk.DeviceArray((1,), np.uint32)
    too_many = 65536 * 1024 + 1  # rejected before any buffer is touched
    rc = L.wrk_compact_noalloc(small.ptr, small.ptr, too_many, small.ptr, count.ptr)
    assert rc == 1  # WRK_ERR_INVALID
    assert b"scratch limit" in L.wrk_last_error()
    # the largest 32-bit size: its tile count must not wrap to zero and pass
    rc = L.wrk_compact_noalloc(small.ptr, small.ptr, 0xFFFFFFFF, small.ptr, count.ptr)
    assert rc == 1
    assert b"scratch limit" in L.wrk_last_error()
    # the empty input is fine and reports zero survivors
    assert L.wrk_compact_noalloc(small.ptr, small.ptr, 0, small.ptr, count.ptr) == 0
    assert int(count.numpy()[0]) == 0
