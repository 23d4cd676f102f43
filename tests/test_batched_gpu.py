"""Batched builds (lvbh_build_batched): many meshes in one launch sequence.

Every mesh's slice of a batched result must equal, word for word, the plain build of that
mesh alone (lvbh_build_soup) and the oracle's build of it: Morton keys, permutation (local to
the mesh), parent links, every BVHNode word and every triangle word, plus the quantisation box.
Sizes cover the tile and block edges of both the sort (4096-key tiles) and the tree pass
(256-leaf blocks), single-triangle and empty meshes.
"""
import numpy as np
import pytest

from test_parity_gpu import FIELDS, assert_same

pytestmark = pytest.mark.gpu

EDGE_SIZES = [1, 2, 3, 0, 64, 255, 256, 257, 511, 4095, 4096, 4097, 8193, 70_001, 1, 0, 300, 12_289]


def make_batch(sizes, seed=11):
    from lvbh import scenes
    rng = np.random.default_rng(seed)
    offs = np.zeros(len(sizes) + 1, dtype=np.int64)
    offs[1:] = np.cumsum(sizes)
    parts = []
    for i, n in enumerate(sizes):
        c = rng.uniform(-100.0, 100.0, (2, 3))
        parts.append(scenes.uniform_soup(int(n), seed=seed * 1000 + i, lo=c.min(0), hi=c.max(0)))
    return np.concatenate(parts) if parts else np.zeros((0, 12), np.float32), offs


def mesh_np(res, i):
    m = res.mesh(i)
    return {"nodes": m.nodes.cpu().numpy().view(np.uint32), "tris": m.tris.cpu().numpy(),
            "parents": m.parents.cpu().numpy(), "leaf_index": m.leaf_index.cpu().numpy().view(np.uint32),
            "morton": m.morton.cpu().numpy().view(np.uint32), "bounds": m.bounds}


def check_against_plain(builder, tri, offs, res, seg_bounds=None):
    import torch
    for i in range(len(offs) - 1):
        a, b = int(offs[i]), int(offs[i + 1])
        hb = None if seg_bounds is None else seg_bounds[i]
        ref = builder.build_soup(torch.from_numpy(np.ascontiguousarray(tri[a:b])).cuda(), hb).to_numpy()
        got = mesh_np(res, i)
        assert_same(got, ref, f"mesh {i} (n={b - a})")
        np.testing.assert_array_equal(got["bounds"].view(np.uint32), ref["bounds"].view(np.uint32),
                                      err_msg=f"mesh {i} bounds")


@pytest.mark.parametrize("graph", [True, False])
def test_batched_edges_match_plain(builder, graph):
    import torch
    tri, offs = make_batch(EDGE_SIZES)
    res = builder.build_batched(torch.from_numpy(tri).cuda(), offs, graph=graph)
    check_against_plain(builder, tri, offs, res)


def test_batched_vs_oracle(builder):
    import torch
    import oracle
    tri, offs = make_batch([1, 2, 257, 4097, 30_000, 3, 9000], seed=5)
    res = builder.build_batched(torch.from_numpy(tri).cuda(), offs)
    for i in range(len(offs) - 1):
        a, b = int(offs[i]), int(offs[i + 1])
        ref = oracle.build(tri[a:b], None, threads=0)
        assert_same(mesh_np(res, i), ref, f"mesh {i}")


def test_batched_host_input_and_host_bounds(builder):
    tri, offs = make_batch([500, 4096, 1, 20_000, 77], seed=9)
    m = len(offs) - 1
    rng = np.random.default_rng(3)
    sb = np.empty((m, 6), np.float32)
    for i in range(m):
        t = tri[offs[i]:offs[i + 1]]
        v = np.concatenate([t[:, 0:3], t[:, 4:7], t[:, 8:11]])
        pad = np.float32(rng.uniform(0.0, 2.0))
        sb[i, :3] = v.min(0) - pad
        sb[i, 3:] = v.max(0) + pad
    res = builder.build_batched(tri, offs, seg_bounds=sb)  # host soup, host per-mesh bounds
    check_against_plain(builder, tri, offs, res, seg_bounds=sb)
    np.testing.assert_array_equal(res.seg_bounds.view(np.uint32), sb.view(np.uint32))


def test_batched_graph_replay_new_table(builder):
    """Two batches with the same totals (same graph shape) but different segment tables: the
    replayed graph must pick up the second table."""
    import torch
    for sizes in ([100, 5000, 300], [5000, 300, 100], [300, 100, 5000]):
        tri, offs = make_batch(sizes, seed=sum(sizes) + sizes[0])
        res = builder.build_batched(torch.from_numpy(tri).cuda(), offs)
        check_against_plain(builder, tri, offs, res)


def test_batched_async_and_reuse(builder):
    import torch
    tri, offs = make_batch([3000, 17, 9000], seed=21)
    t = torch.from_numpy(tri).cuda()
    r1 = builder.build_batched(t, offs, sync=False)
    builder.sync()
    r2 = builder.build_batched(t, offs)
    for f in FIELDS:
        assert torch.equal(getattr(r1, f), getattr(r2, f)), f
    np.testing.assert_array_equal(r1.seg_bounds, r2.seg_bounds)


def test_batched_mesh_batch_sample(builder):
    """A 64-mesh sample of the batched workload's generator (log-uniform sizes in
    [64, 262144], random boxes) against per-mesh plain builds."""
    import torch
    from lvbh import scenes
    tri, offs = scenes.mesh_batch(count=64, seed=3)
    res = builder.build_batched(torch.from_numpy(tri).cuda(), offs, profile=True)
    assert set(res.stage_ms) == {"upload", "bounds", "morton", "sort", "gather", "tree", "top"}
    check_against_plain(builder, tri, offs, res)


def test_batched_rejects_bad_offsets(builder):
    import lvbh
    import torch
    t = torch.zeros((10, 12), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError):
        builder.build_batched(t, [1, 10])
    with pytest.raises(ValueError):
        builder.build_batched(t, [0, 6, 4, 10])
    with pytest.raises(ValueError):
        builder.build_batched(t, [0, 9])
    # the C ABI checks the same rules itself
    import ctypes
    L = lvbh._native.lib
    offs = np.array([0, 6, 4, 10], dtype=np.uint32)
    r = lvbh._native.Result()
    rc = L.lvbh_build_batched(builder.ctx, ctypes.c_void_p(t.data_ptr()),
                              offs.ctypes.data_as(ctypes.c_void_p), 3, None, None,
                              lvbh._native.OUT_CALLER, ctypes.byref(r), None)
    assert rc == lvbh._native.EINVAL


def test_batched_empty(builder):
    import torch
    res = builder.build_batched(torch.zeros((0, 12), dtype=torch.float32, device="cuda"), [0, 0, 0])
    assert res.nodes.shape[0] == 0
    np.testing.assert_array_equal(res.seg_bounds, np.zeros((2, 6), np.float32))


@pytest.mark.parametrize("digit_bits,tree_block", [(10, 256), (10, 128), (8, 256), (8, 128)])
def test_batched_every_tunable_choice_is_identical(builder, digit_bits, tree_block):
    import torch
    tri, offs = make_batch(EDGE_SIZES, seed=31)
    builder.set_tunables(digit_bits=digit_bits, tree_block=tree_block)
    try:
        res = builder.build_batched(torch.from_numpy(tri).cuda(), offs)
        t = builder.tunables()
        assert (t["digit_bits"], t["tree_block"]) == (digit_bits, tree_block)
    finally:
        builder.set_tunables()
    check_against_plain(builder, tri, offs, res)


def test_autotune_times_candidates_and_caches(builder):
    import torch
    from lvbh import scenes
    tri, offs = scenes.mesh_batch(count=96, seed=8)
    t = torch.from_numpy(tri).cuda()
    r1 = builder.build_batched(t, offs, autotune=True)
    first = builder.tunables()
    assert len(first["candidates_ms"]) == 4 and min(first["candidates_ms"]) > 0
    cands = [(10, 256), (10, 128), (8, 256), (8, 128)]
    best = cands[int(np.argmin(first["candidates_ms"]))]
    assert (first["digit_bits"], first["tree_block"]) == best
    r2 = builder.build_batched(t, offs, autotune=True)  # same histogram: cached, not re-timed
    again = builder.tunables()
    assert again == first
    for f in FIELDS:
        assert torch.equal(getattr(r1, f), getattr(r2, f)), f
    check_against_plain(builder, tri, offs, r2)


def test_async_batched_then_larger_batch_keeps_first_status_and_bounds():
    """An LVBH_ASYNC batched build followed, without lvbh_sync, by a larger batched build on the
    same context (through the C ABI: the Python wrapper syncs in between by itself).  The second
    call grows the batch scratch and its pinned mirror; it must first finish the pending build,
    so that the first build's per-mesh bounds reach its bounds_out intact."""
    import ctypes

    import torch
    import lvbh
    import oracle
    from lvbh import _native
    L = _native.lib
    b = lvbh.BVHBuilder(0)
    try:
        calls = []
        for sizes, seed in (([300, 5000, 17, 4096], 61), ([900, 70_001, 3, 12_289, 40_000, 8, 4097, 256], 62)):
            tri, offs = make_batch(sizes, seed=seed)
            n, m = int(offs[-1]), len(sizes)
            dtri = torch.from_numpy(tri).cuda()
            outs = lvbh.empty_outputs(n, dtri.device)
            r = lvbh._result_struct(outs, n)
            offs32 = offs.astype(np.uint32)
            bout = np.full((m, 6), np.nan, np.float32)
            rc = L.lvbh_build_batched(b.ctx, ctypes.c_void_p(dtri.data_ptr()),
                                      offs32.ctypes.data_as(ctypes.c_void_p), m, None,
                                      bout.ctypes.data_as(ctypes.c_void_p),
                                      _native.OUT_CALLER | _native.ASYNC, ctypes.byref(r), None)
            assert rc == _native.OK, L.lvbh_last_error(b.ctx)
            calls.append((tri, offs, bout, outs, dtri, r, offs32))
        assert L.lvbh_sync(b.ctx) == _native.OK
        for tri, offs, bout, outs, *_ in calls:
            for i in range(len(offs) - 1):
                t = tri[offs[i]:offs[i + 1]]
                np.testing.assert_array_equal(bout[i].view(np.uint32), oracle.scene_bounds(t).view(np.uint32),
                                              err_msg=f"mesh {i} bounds_out")
                ref = oracle.build(t, None, threads=0)
                a, c = int(offs[i]), int(offs[i + 1])
                got = {"nodes": outs["nodes"][a:c].cpu().numpy().view(np.uint32),
                       "tris": outs["tris"][a:c].cpu().numpy(),
                       "parents": outs["parents"][2 * a:2 * c].cpu().numpy(),
                       "leaf_index": outs["leaf_index"][a:c].cpu().numpy().view(np.uint32),
                       "morton": outs["morton"][a:c].cpu().numpy().view(np.uint32)}
                assert_same(got, ref, f"mesh {i}")
    finally:
        b.close()


def test_lookback_wait_runs_out_then_clean_build(builder):
    """A device wait that runs out, made on the host side: with the test hook, sort tile 1 (the
    second tile of mesh 0) never publishes its look-back counts, so the later tiles of mesh 0
    wait until their lowered bound (2e6 cycles, about a millisecond) runs out.  The build must
    report LVBH_ETIMEOUT, build no tree from the unfinished sort, and leave the context usable:
    the next build on it, hook cleared, equals the build on an untouched context."""
    import time
    import torch
    import lvbh
    import lvbh._native as nat
    tri, offs = make_batch([20_000, 300, 9000], seed=21)  # mesh 0 spans sort tiles 0..4
    t = torch.from_numpy(tri).cuda()
    ref = builder.build_batched(t, offs)
    b = lvbh.BVHBuilder(0)
    try:
        assert nat.lib.lvbh_test_stall_lookback(b.ctx, 1, 2_000_000) == nat.OK
        t0 = time.perf_counter()
        with pytest.raises(nat.LvbhError) as ei:
            b.build_batched(t, offs)
        assert ei.value.code == nat.ETIMEOUT, str(ei.value)
        assert "look-back" in str(ei.value)
        assert time.perf_counter() - t0 < 5.0
        assert nat.lib.lvbh_test_stall_lookback(b.ctx, 0xFFFFFFFF, 0) == nat.OK
        got = b.build_batched(t, offs)
        for i in range(len(offs) - 1):
            assert_same(mesh_np(got, i), mesh_np(ref, i), f"mesh {i} after the timed-out build")
    finally:
        b.close()
