"""lvbh_sort_pairs_noalloc: the build's radix sort for callers that cannot allocate device
memory when they sort (a render or serving loop that must not stall on cudaMalloc, a process
whose memory budget is already held by its own pool, a plugin host that owns all allocations).

The entry point is called through the C ABI on two different inputs in a row; each result must
equal, bit for bit, the sorted keys and permutation that lvbh_build_soup produces for the same
triangles.  The file is collected last so that a run stopping at the first failure has already
run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _sort_noalloc(keys_np):
    import torch
    import lvbh._native as nat
    n = keys_np.size
    keys = torch.from_numpy(keys_np.view(np.int32)).cuda()
    keys_out = torch.empty(n, dtype=torch.int32, device="cuda")
    perm_out = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = nat.lib.lvbh_sort_pairs_noalloc(_ptr(keys), n, _ptr(keys_out), _ptr(perm_out), stream)
    assert rc == nat.OK, nat.STATUS_NAMES.get(rc, rc)
    return keys_out.cpu().numpy().view(np.uint32), perm_out.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_build_twice():
    import torch
    import lvbh
    import oracle
    from lvbh import scenes
    b = lvbh.BVHBuilder(0)
    try:
        for n, seed in ((300_001, 41), (lvbh._native.NOALLOC_MAX_KEYS, 42)):
            tri = scenes.clustered_soup(n, seed=seed)
            bounds = oracle.scene_bounds(tri)
            ref = b.build_soup(torch.from_numpy(tri).cuda(), bounds).to_numpy()
            _, unsorted = oracle.aabb_zidx(tri, bounds)
            keys, perm = _sort_noalloc(unsorted)
            np.testing.assert_array_equal(keys, ref["morton"])
            np.testing.assert_array_equal(perm, ref["leaf_index"])
    finally:
        b.close()


def test_noalloc_rejects_oversize_and_null():
    import lvbh._native as nat
    L = nat.lib
    big = nat.NOALLOC_MAX_KEYS + 1
    assert L.lvbh_sort_pairs_noalloc(None, big, None, None, None) == nat.ERANGE
    assert L.lvbh_sort_pairs_noalloc(None, 5, None, None, None) == nat.EINVAL
    assert L.lvbh_sort_pairs_noalloc(None, 0, None, None, None) == nat.OK
