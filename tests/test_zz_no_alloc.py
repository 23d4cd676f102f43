"""lvbh_sort_pairs_noalloc: the build's radix sort for callers that cannot allocate device
memory when they sort (a render or serving loop that must not stall on cudaMalloc, a process
whose memory budget is already held by its own pool, a plugin host that owns all allocations).

The entry point is called through the C ABI on two different inputs in a row; each result must
equal, bit for bit, the sorted keys and permutation that lvbh_build_soup produces for the same
triangles.  Full-range 32-bit keys (all four 8-bit digits in use, duplicates, the extremes) are
checked against numpy's stable argsort, largest size first, and the sort also runs in place.  The file is collected last so that a run stopping at the first failure has already
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


def _full_range_cases(n, seed):
    """Full 32-bit keys the build never produces: uniform over all 2^32 values with 0 and
    0xFFFFFFFF planted, keys that differ only in bits 30-31, and long runs of equal keys."""
    rng = np.random.default_rng(seed)
    uni = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    uni[rng.integers(0, n, 64)] = 0xFFFFFFFF
    uni[rng.integers(0, n, 64)] = 0
    top = (rng.integers(0, 4, n, dtype=np.uint32) << np.uint32(30)) | np.uint32(0x155)
    runs = np.repeat(rng.integers(0, 1 << 32, n // 5000 + 1, dtype=np.uint64).astype(np.uint32), 5000)[:n]
    runs[rng.random(n) < 0.1] = 0xFFFFFFFF
    return {"uniform": uni, "top_bits": top, "runs": runs}


def test_noalloc_full_range_keys_max_then_small():
    """Against the stable argsort on full-range keys; the largest size first, then a smaller
    size that is not a multiple of the 4096-key tile, so look-back words and tile counters
    left by the larger call would show if they leaked into the next one."""
    nmax = __import__("lvbh")._native.NOALLOC_MAX_KEYS
    for n, seed in ((nmax, 7), (1000, 8), (nmax - 4095, 9), (4097, 10)):
        for name, keys in _full_range_cases(n, seed).items():
            got_k, got_p = _sort_noalloc(keys)
            order = np.argsort(keys, kind="stable").astype(np.uint32)
            np.testing.assert_array_equal(got_p, order, err_msg=f"{name} n={n} perm")
            np.testing.assert_array_equal(got_k, keys[order], err_msg=f"{name} n={n} keys")


def test_noalloc_in_place():
    """keys_out may be the input array itself (keys_in is read only before keys_out is first
    written)."""
    import ctypes
    import torch
    import lvbh._native as nat
    keys = _full_range_cases(300_000, 12)["uniform"]
    t = torch.from_numpy(keys.view(np.int32)).cuda()
    perm = torch.empty_like(t)
    rc = nat.lib.lvbh_sort_pairs_noalloc(_ptr(t), keys.size, _ptr(t), _ptr(perm),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == nat.OK
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    np.testing.assert_array_equal(perm.cpu().numpy().view(np.uint32), order)
    np.testing.assert_array_equal(t.cpu().numpy().view(np.uint32), keys[order])


def test_noalloc_rejects_oversize_and_null():
    import lvbh._native as nat
    L = nat.lib
    big = nat.NOALLOC_MAX_KEYS + 1
    assert L.lvbh_sort_pairs_noalloc(None, big, None, None, None) == nat.ERANGE
    assert L.lvbh_sort_pairs_noalloc(None, 5, None, None, None) == nat.EINVAL
    assert L.lvbh_sort_pairs_noalloc(None, 0, None, None, None) == nat.OK
