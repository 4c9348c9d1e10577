"""spb_intersect_host_static: the closest-hit entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc (cudaMalloc may synchronize the device and
may fail when memory runs out, so a frame loop with a fixed time budget or an application
whose allocator owns all device memory must not allocate per call).  It stages rays and
results in a fixed device array the library reserves at load time, so its answers must equal
those of spb_intersect_host, which stages through buffers it allocates -- on every call,
including consecutive calls that reuse the array -- and it must take no device memory.  This file is collected last so that a run
stopping at its first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

import sprout_b200 as sb
from sprout_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536  # SPB_STATIC_MAX_RAYS in include/sprout_b200.h


def _static_cast(tree, rays):
    lib = _lib.load()
    n = rays.shape[0]
    ids = np.full(n, 0xDEADBEEF, np.uint32)
    ts = np.full(n, np.nan, np.float32)
    status = lib.spb_intersect_host_static(tree._handle, rays.ctypes.data, n, ids.ctypes.data, ts.ctypes.data)
    return status, ids, ts


def test_static_scratch_cast_matches_allocating_cast_twice_in_a_row():
    pos, idx = sb.sphere_mesh(64, 0.1, 1)
    with sb.Tree() as tree:
        tree.build(pos, idx)
        for seed in (21, 22):  # two consecutive calls through the shared array
            rays = sb.random_rays(40000, seed=seed)
            want_ids, want_t = tree.intersect(rays)
            status, ids, ts = _static_cast(tree, rays)
            assert status == 0, _lib.load().spb_last_error()
            assert np.array_equal(ids, want_ids)
            assert np.array_equal(ts.view(np.uint32), want_t.view(np.uint32))
        assert (want_ids != sb.MISS).any()


def test_static_scratch_cast_allocates_nothing_on_a_fresh_tree():
    """The property that sets this entry point apart: on a freshly built tree that has never
    cast, a static call leaves the device's free memory (cudaMemGetInfo) unchanged, while the
    allocating entry point's first call on the same tree visibly takes its staging buffers --
    which shows the check would see an allocation.  Only then are the answers compared."""
    import torch

    pos, idx = sb.sphere_mesh(64, 0.1, 1)
    rays = sb.random_rays(50000, seed=31)
    with sb.Tree() as first:
        # The first static call in a process looks up the array's device address.
        first.build(pos, idx)
        assert _static_cast(first, rays[:16])[0] == 0
    with sb.Tree() as tree:
        tree.build(pos, idx)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        status, ids, ts = _static_cast(tree, rays)
        free_after = torch.cuda.mem_get_info()[0]
        assert status == 0, _lib.load().spb_last_error()
        assert free_after == free_before
        want_ids, want_t = tree.intersect(rays)
        assert torch.cuda.mem_get_info()[0] < free_after
        assert tree.status() == 0
    assert np.array_equal(ids, want_ids)
    assert np.array_equal(ts.view(np.uint32), want_t.view(np.uint32))


def test_static_scratch_cast_rejects_batches_beyond_its_limit():
    pos, idx = sb.sphere_mesh(8, 0.1, 1)
    with sb.Tree() as tree:
        tree.build(pos, idx)
        rays = sb.random_rays(MAX_RAYS + 1, seed=3)
        status, _, _ = _static_cast(tree, rays)
        assert status == _lib.SPB_ERROR_ARGUMENT
        assert b"static scratch limit" in _lib.load().spb_last_error()
        # the largest accepted batch still works
        status, ids, _ = _static_cast(tree, rays[:MAX_RAYS])
        assert status == 0
        assert np.array_equal(ids, tree.intersect(rays[:MAX_RAYS])[0])
